"""The sharded step's host logic on the CPU, with the oracle as each rank's
stepper: the Morton split, the sub-meshes and their halo plans, and the step
protocol (exchange, step, minimum of dt) give the owned cells bit for bit as
a single-domain run, both with the ranks emulated in one process and as two
gloo ranks over torch.distributed."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import oracle_lib as ol


def _problem(titan, **kw):
    m, p, st, _ = titan.problems.heliosphere_shell(nq=6, nlayer=6, move=True, **kw)
    return m, p, np.ascontiguousarray(st)


class OracleStepper:
    """The oracle on a sub-mesh, with the interface of shard.DeviceStepper."""

    def __init__(self, pkg, mesh, params):
        self.run = ol.OracleRun(mesh, params)
        self.state = None
        self.send = self.recv = None

    @property
    def dt(self):
        return float(self.run.clock[0])

    @dt.setter
    def dt(self, v):
        self.run.clock[0] = v

    def set_halo(self, send, recv):
        self.send, self.recv = np.asarray(send), np.asarray(recv)

    def set_face_method(self, m):
        self.run.set_face_method(m)

    def set_cfl_faces(self, exclude):
        self.run.set_cfl_faces(exclude)

    def pack(self, buf):
        buf[: len(self.send)] = torch.from_numpy(np.ascontiguousarray(self.state[:, self.send].T[:, : buf.shape[1]]))

    def unpack(self, buf):
        self.state[: buf.shape[1], self.recv] = buf[: len(self.recv)].numpy().T

    def upload_state(self, st):
        self.state = np.ascontiguousarray(st.copy())

    def download_state(self):
        return self.state.copy()

    def go(self, n):
        assert self.run.go(self.state, n).err_code == 0

    def close(self):
        pass


def test_sub_meshes_and_plans_are_consistent(titan):
    m, _, _ = _problem(titan)
    S = titan.shard
    for world in (2, 3, 5):
        owner = S.partition(m, world)
        assert np.bincount(owner, minlength=world).min() > 0
        shards = [S.build_shard(m, owner, r) for r in range(world)]
        for r, sh in enumerate(shards):
            lm, n_own = sh["mesh"], sh["n_owned"]
            assert (owner[sh["cells"][:n_own]] == r).all() and (owner[sh["cells"][n_own:]] != r).all()
            # every face of an owned cell keeps both its cells (or its true boundary)
            f_own = np.unique(lm["cell_faces"][:n_own])
            g = sh["faces"][f_own]
            assert np.array_equal(lm["face_type"][f_own], m["face_type"][g])
            both = m["face_cells"][g]
            for k in (0, 1):
                loc = lm["face_cells"][f_own, k]
                assert np.array_equal(np.where(loc >= 0, sh["cells"][np.maximum(loc, 0)], -1), both[:, k])
            # what r sends to q is what q receives from r, cell for cell
            for q, ids in sh["send"].items():
                assert np.array_equal(sh["cells"][ids], shards[q]["cells"][shards[q]["recv"][r]])


def _emulated(titan, world, steps, **kw):
    m, p, st = _problem(titan, **kw)
    S = titan.shard
    owner = S.partition(m, world)
    ranks = []
    layers = 2 if p["tvd"] else 1
    for r in range(world):
        sh = S.build_shard(m, owner, r, layers=layers)
        o = OracleStepper(None, sh["mesh"], p)
        o.set_cfl_faces(sh["nodt"])
        o.upload_state(st[:, sh["cells"]])
        ranks.append((sh, o))
    full = ol.OracleRun(m, p)
    ref = st.copy()
    for _ in range(steps):
        # owners' states into the copies, step every rank, the minimum dt
        for r, (sh, o) in enumerate(ranks):
            for q, ids in sh["recv"].items():
                shq, oq = ranks[q]
                o.state[:, ids] = oq.state[:, shq["send"][r]]
        for sh, o in ranks:
            o.go(1)
        dt = min(o.dt for _, o in ranks)
        for _, o in ranks:
            o.dt = dt
        assert full.go(ref, 1).err_code == 0
        assert full.clock[0] == dt
    return ranks, ref


@pytest.mark.parametrize("world,kw", [(2, {}), (4, {}), (3, dict(tvd=True, zones=True, npassive=2))])
def test_emulated_ranks_match_the_single_domain_step_bit_for_bit(titan, oracle_lib, world, kw):
    ranks, ref = _emulated(titan, world, 4, **kw)
    for sh, o in ranks:
        n = sh["n_owned"]
        assert np.array_equal(o.state[:, :n], ref[:, sh["cells"][:n]])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import importlib
    import sys

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        titan = importlib.import_module("titan_c-_b200")
        m, p, st = _problem(titan)
        ss = titan.shard.ShardedStep(titan, m, p, rank, world, torch.device("cpu"), stepper=OracleStepper)
        ss.upload_state(st)
        ss.go(3)
        own = ss.owned_state()
        full = np.zeros_like(st)
        full[:, ss.shard["cells"][: ss.shard["n_owned"]]] = own
        t = torch.from_numpy(full)
        torch.distributed.all_reduce(t)          # owned cells are disjoint
        if rank == 0:
            out.put((t.numpy(), ss.step.dt))
    finally:
        torch.distributed.destroy_process_group()


def test_two_gloo_ranks_match_the_single_domain_step(titan, oracle_lib):
    m, p, st = _problem(titan)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    got, dt = q.get(timeout=240)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    full = ol.OracleRun(m, p)
    ref = st.copy()
    assert full.go(ref, 3).err_code == 0
    assert np.array_equal(got[:8], ref[:8])
    assert dt == full.clock[0]


def _gloo_rank_that_may_fail(rank, world, port, out, fail_rank):
    """Rank `fail_rank` leaves after the set-up barrier, between steps, with none
    of its exchanges in flight; the others must end their next step with an
    error within the process group's timeout instead of waiting for good."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import importlib
    import sys
    import time

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=10))
    titan = importlib.import_module("titan_c-_b200")
    m, p, st = _problem(titan)
    ss = titan.shard.ShardedStep(titan, m, p, rank, world, torch.device("cpu"), stepper=OracleStepper)
    ss.upload_state(st)
    if rank == fail_rank:
        os._exit(3)  # the rank dies between steps
    t0 = time.monotonic()
    try:
        ss.go(3)
        out.put((rank, "no error", time.monotonic() - t0))
    except Exception as e:  # noqa: BLE001 - any error the collective raises
        out.put((rank, type(e).__name__, time.monotonic() - t0))
    out.close()
    out.join_thread()  # the queue's feeder thread has written the result
    os._exit(0)


def test_a_rank_that_dies_between_steps_ends_the_others_with_an_error(titan):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank_that_may_fail, args=(r, 2, port, q, 1)) for r in range(2)]
    for pr in procs:
        pr.start()
    rank, what, waited = q.get(timeout=240)
    for pr in procs:
        pr.join(timeout=60)
    assert rank == 0 and what != "no error"
    assert waited < 60.0
    assert procs[1].exitcode == 3 and procs[0].exitcode == 0
