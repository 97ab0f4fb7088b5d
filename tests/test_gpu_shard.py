"""The sharded step's device side on one GPU: two contexts on the two halves
of a shell (titan.shard sub-meshes), their halo cells moved through device
buffers by titan_pack_halo / titan_unpack_halo, stepped one after the other
with the minimum dt, give the owned cells bit for bit as one context on the
whole shell. (Ranks on separate GPUs move the same buffers with NCCL; the
CPU tests run that protocol with gloo.)"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

NET = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "titan_c-_b200", "data",
                   "closure_shell.npz")


@pytest.mark.parametrize("world,kw,closure", [(2, {}, False), (3, {}, False), (3, dict(tvd=True, zones=True), False),
                                              (2, dict(flux_precision=32), True)])
def test_contexts_exchanging_halos_match_one_context(titan, world, kw, closure):
    """closure: the mixed step with the trained network's sources, per rank on
    its own cells (each cell's sources depend on that cell alone)."""
    m, p, st, _ = titan.problems.heliosphere_shell(nq=8, nlayer=8, move=True, npassive=2, **kw)
    S = titan.shard
    dev = torch.device("cuda:0")
    net = titan.closure.Closure.load(NET) if closure else None
    owner = S.partition(m, world)
    ranks = []
    for r in range(world):
        sh = S.build_shard(m, owner, r, layers=2 if p["tvd"] else 1)
        step = titan.PlasmaStep(sh["mesh"], p)
        step.set_cfl_faces(sh["nodt"])
        if net is not None:
            net.install(step)
        step.upload_state(np.ascontiguousarray(st[:, sh["cells"]]))
        bufs = {q: torch.empty((len(ids), 10), dtype=torch.float64, device=dev) for q, ids in sh["send"].items()}
        ranks.append((sh, step, bufs))
    ns = 8 + p["npassive"]
    full = titan.PlasmaStep(m, p)
    if net is not None:
        net.install(full)
    full.upload_state(st)
    for _ in range(6):
        # every rank packs what each peer needs, then unpacks what it receives
        for sh, step, bufs in ranks:
            for q, ids in sh["send"].items():
                step.set_halo(ids, np.zeros(0, np.int32))
                step.pack_halo(bufs[q].data_ptr())
        torch.cuda.synchronize()  # packs are ordered on each context's own stream
        for r, (sh, step, _) in enumerate(ranks):
            for q, ids in sh["recv"].items():
                src = ranks[q][2][r]
                step.set_halo(np.zeros(0, np.int32), ids)
                step.unpack_halo(src.data_ptr())
        torch.cuda.synchronize()
        for sh, step, _ in ranks:
            step.go(1)
        dt = min(step.dt for _, step, _ in ranks)
        for _, step, _ in ranks:
            step.dt = dt
        full.go(1)
        assert full.dt == dt
    ref = full.download_state()
    for sh, step, _ in ranks:
        n = sh["n_owned"]
        got = step.download_state()[:ns, :n]
        assert np.array_equal(got, ref[:ns, sh["cells"][:n]])
        step.close()
    full.close()


def test_pack_unpack_round_trip(titan):
    m, p, st, _ = titan.problems.heliosphere_shell(nq=6, nlayer=6, move=False)
    g = titan.PlasmaStep(m, p)
    g.upload_state(st)
    ids = np.arange(0, g.ncell, 7, dtype=np.int32)
    buf = torch.empty((len(ids), 8), dtype=torch.float64, device="cuda:0")
    g.set_halo(ids, ids[::-1].copy())
    g.pack_halo(buf.data_ptr())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(buf.cpu().numpy(), st[:8, ids].T)
    g.unpack_halo(buf.data_ptr())                 # the same cells, in reverse order
    got = g.download_state()
    np.testing.assert_array_equal(got[:8, ids[::-1]], st[:8, ids])
    with pytest.raises(titan.native.TitanError):
        g.set_halo(np.array([g.ncell], np.int32), np.zeros(0, np.int32))
    g.close()


def test_device_paced_contexts_match_one_context(titan):
    """The loop paced by the device (titan_set_clock, titan_step_async,
    titan_dt_copy, titan_get_clock) with two contexts on one GPU: each step's
    packs, unpacks and steps run on the contexts' own streams, ordered by
    events only, and dt is the minimum formed on the device; the host waits
    once, at the end. The owned cells, dt and t equal one context's."""
    m, p, st, _ = titan.problems.heliosphere_shell(nq=8, nlayer=8, move=True, npassive=2)
    S = titan.shard
    dev = torch.device("cuda:0")
    world = 2
    owner = S.partition(m, world)
    ranks = []
    for r in range(world):
        sh = S.build_shard(m, owner, r)
        step = titan.PlasmaStep(sh["mesh"], p)
        step.set_cfl_faces(sh["nodt"])
        step.upload_state(np.ascontiguousarray(st[:, sh["cells"]]))
        ids = {q: ids for q, ids in sh["send"].items()}
        bufs = {q: torch.empty((len(i), 10), dtype=torch.float64, device=dev) for q, i in ids.items()}
        stream = torch.cuda.ExternalStream(step.stream(), device=dev)
        ranks.append(dict(sh=sh, step=step, bufs=bufs, stream=stream, dt=torch.zeros(1, dtype=torch.float64,
                                                                                     device=dev)))
    full = titan.PlasmaStep(m, p)
    full.upload_state(st)
    steps = 6
    for R in ranks:
        R["step"].set_clock(1e-5, 0.0)
    for _ in range(steps):
        packed = []
        for R in ranks:
            for q, ids in R["sh"]["send"].items():
                R["step"].set_halo(ids, np.zeros(0, np.int32))
                R["step"].pack_halo(R["bufs"][q].data_ptr())
            ev = torch.cuda.Event()
            ev.record(R["stream"])
            packed.append(ev)
        for r, R in enumerate(ranks):
            for q, ids in R["sh"]["recv"].items():
                R["stream"].wait_event(packed[q])
                R["step"].set_halo(np.zeros(0, np.int32), ids)
                R["step"].unpack_halo(ranks[q]["bufs"][r].data_ptr())
            R["step"].step_async(1)
            R["step"].dt_copy(R["dt"].data_ptr(), into_clock=False)
        # the minimum of dt over the contexts, on the device, back into every clock
        done = []
        for R in ranks:
            ev = torch.cuda.Event()
            ev.record(R["stream"])
            done.append(ev)
        for R in ranks:
            for ev in done:
                R["stream"].wait_event(ev)
            with torch.cuda.stream(R["stream"]):
                R["dt_min"] = torch.minimum(ranks[0]["dt"], ranks[1]["dt"])
            R["step"].dt_copy(R["dt_min"].data_ptr(), into_clock=True)
        full.go(1)
    ref = full.download_state()
    for R in ranks:
        info = R["step"].get_clock()
        assert info["steps_done"] == steps
        assert R["step"].dt == full.dt and R["step"].t == full.t
        n = R["sh"]["n_owned"]
        got = R["step"].download_state()[:10, :n]
        assert np.array_equal(got, ref[:10, R["sh"]["cells"][:n]])
        R["step"].close()
    full.close()


def test_sharded_step_paced_by_the_device_over_nccl(titan):
    """ShardedStep's device-paced loop through torch.distributed with NCCL, one
    rank: its dt all-reduce runs on the context's stream; the result equals
    one context's steps."""
    import socket

    import torch.distributed as dist

    m, p, st, _ = titan.problems.heliosphere_shell(nq=8, nlayer=8, move=True)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        dev = torch.device("cuda:0")
        ss = titan.shard.ShardedStep(titan, m, p, 0, 1, dev)
        ss.upload_state(st)
        ss.go(3)
        ss.go(2)
        got = ss.owned_state()
        cells = ss.shard["cells"][:ss.shard["n_owned"]]
        dt = ss.step.dt
        ss.close()
    finally:
        dist.destroy_process_group()
    full = titan.PlasmaStep(m, p)
    full.upload_state(st)
    full.go(3)
    full.go(2)
    ref = full.download_state()
    assert full.dt == dt
    assert np.array_equal(got[:8], ref[:8, cells])
    full.close()
