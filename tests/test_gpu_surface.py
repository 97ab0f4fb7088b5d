"""Surface-tracking node motion on the GPU (titan_set_surface_motion:
Setka::Culc_Velocity_surface, TITAN/source/Setka_move.cpp:111-1358, and
Luch::dvigenie, Luch.cpp:6-739) against the oracle, step by step: the nodes
and the state after each step within the contract's 1e-12 relative, with TS,
HP and BS surfaces moving on a shell, and with the options that change the
HP faces (null_bn_on_HP, bn_in_p_on_HP), second-order faces, passive
scalars, rays of different lengths and the smoothing terms (sglag_*). The exact HP solver calls pow, which CUDA and glibc may round
differently by an ulp."""
import numpy as np
import pytest

import oracle_lib as ol
from test_gpu_parity import REL, rel_err

pytestmark = pytest.mark.gpu

SURF = dict(velocity_TS=1.0, velocity_HP=1.0, velocity_BS=1.0, move_TS=1, move_HP=1, move_BS=1, null_bn_on_HP=0)


def _surface_shell(T, **kw):
    m, p, st, _ = T.problems.heliosphere_shell(nq=8, nlayer=12, move=True, **kw)
    for layer, kind in ((7, 1), (9, 2), (11, 3)):
        T.mesh.mark_shell_surface(m, layer, kind)
    return m, p, st, T.mesh.shell_rays(m)


@pytest.mark.parametrize("variant", [
    dict(),
    dict(surface=dict(null_bn_on_HP=1)),
    dict(params=dict(bn_in_p_on_hp=1)),
    dict(shell=dict(tvd=True, zones=True, npassive=2), surface=dict(velocity_HP=0.5)),
    dict(ragged=True),
    dict(surface=dict(sglag_TS=1, sglag_HP=1, sglag_BS=1, sglag_TS_k_sphere=0.3, sglag_HP_k_sphere=0.3,
                      sglag_BS_k=0.3, null_bn_on_HP=1)),
    dict(surface=dict(hp_tail=1)),
])
def test_surface_tracking_steps_match_oracle(titan, oracle_lib, variant):
    m, p, st, rays = _surface_shell(titan, **variant.get("shell", {}))
    if variant.get("ragged"):
        rays[::2, -1] = -1          # every other ray one node shorter: its outer node stays put
    p = dict(p, **variant.get("params", {}))
    surf = dict(SURF, **variant.get("surface", {}))
    gpu = titan.PlasmaStep(m, p)
    gpu.set_surface_motion(rays, **surf)
    run = ol.OracleRun(m, p, surface=surf, rays=rays)
    gpu.upload_state(st)
    x0 = gpu.nodes()
    ns = 8 + p["npassive"]
    worst_s = worst_x = 0.0
    for _ in range(8):
        before = np.ascontiguousarray(gpu.download_state())
        run.xyz[:] = gpu.nodes()
        run.clock[:] = (gpu.dt, gpu.t)
        gpu.go(1)
        assert run.go(before, 1).err_code == 0
        worst_s = max(worst_s, rel_err(gpu.download_state()[:ns], before[:ns]))
        x = gpu.nodes()
        worst_x = max(worst_x, float(np.abs(x - run.xyz).max() / np.abs(run.xyz).max()))
    assert worst_s <= REL, worst_s
    assert worst_x <= REL, worst_x
    # the surfaces did move, the rays' ends did not
    x = gpu.nodes()
    r0, r1 = np.linalg.norm(x0[rays], axis=2), np.linalg.norm(x[rays], axis=2)
    assert np.abs(r1[:, [7, 9, 11]] - r0[:, [7, 9, 11]]).max() > 0
    assert np.array_equal(x[rays[:, 0]], x0[rays[:, 0]])
    full = rays[:, -1] >= 0
    assert np.array_equal(x[rays[full, -1]], x0[rays[full, -1]])
    if surf.get("hp_tail"):
        # the heliotail's HP nodes move across the x axis only
        hp = rays[:, 9]
        tail = x0[hp, 0] < 0
        assert tail.any() and np.array_equal(x[hp[tail], 0], x0[hp[tail], 0])
    gpu.close()


def test_graph_steps_equal_single_steps(titan):
    m, p, st, rays = _surface_shell(titan)
    out = []
    for chunks in ([6], [1] * 6):
        g = titan.PlasmaStep(m, p)
        g.set_surface_motion(rays, **SURF)
        g.upload_state(st)
        for k in chunks:
            g.go(k)
        out.append((g.download_state(), g.nodes()))
        g.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_back_to_prescribed_motion_and_bad_rays(titan):
    m, p, st, rays = _surface_shell(titan)
    g = titan.PlasmaStep(m, p)
    bad = rays.copy()
    bad[1, 3] = bad[0, 3]                      # a node on two rays
    with pytest.raises(titan.native.TitanError):
        g.set_surface_motion(bad, **SURF)
    g.set_surface_motion(rays, **SURF)
    g.set_surface_motion(None)                  # the prescribed radial law again
    g.upload_state(st)
    g.go(2)
    assert np.isfinite(g.download_state()).all()
    g.close()


def test_a_luch_ray_law_steps_match_oracle(titan, oracle_lib):
    """The A_Luch spacing law (titan_set_ray_law, Luch.cpp:9-152) on a shell
    built by that law: nodes and state after each step within 1e-12 of the
    oracle; a ray of the wrong length or without a surface node on the law's
    slots is refused."""
    from test_oracle_surface import LAW, LAW_SLOTS, law_shell

    m, p, st, rays = law_shell(titan, nq=8)
    surf = dict(SURF, velocity_TS=30.0, velocity_HP=30.0, velocity_BS=30.0)
    gpu = titan.PlasmaStep(m, p)
    gpu.set_surface_motion(rays, **surf)
    gpu.set_ray_law(LAW)
    run = ol.OracleRun(m, p, surface=surf, rays=rays, ray_law=LAW)
    gpu.upload_state(st)
    x0 = gpu.nodes()
    worst_s = worst_x = 0.0
    for _ in range(6):
        before = np.ascontiguousarray(gpu.download_state())
        run.xyz[:] = gpu.nodes()
        run.clock[:] = (gpu.dt, gpu.t)
        gpu.go(1)
        assert run.go(before, 1).err_code == 0
        worst_s = max(worst_s, rel_err(gpu.download_state()[:8], before[:8]))
        worst_x = max(worst_x, float(np.abs(gpu.nodes() - run.xyz).max() / np.abs(run.xyz).max()))
    assert worst_s <= REL, worst_s
    assert worst_x <= REL, worst_x
    x = gpu.nodes()
    r0, r1 = np.linalg.norm(x0[rays], axis=2), np.linalg.norm(x[rays], axis=2)
    assert np.abs(r1[:, list(LAW_SLOTS)] - r0[:, list(LAW_SLOTS)]).max() > 1e-6
    # the graph path (several steps per call) gives the same nodes
    g2 = titan.PlasmaStep(m, p)
    g2.set_surface_motion(rays, **surf)
    g2.set_ray_law(LAW)
    g2.upload_state(st)
    g2.go(6)
    assert np.array_equal(g2.nodes(), x)
    g2.close()
    # a law whose ray length differs, or whose TS slot holds no TS node, is refused
    with pytest.raises(titan.TitanError):
        gpu.set_ray_law(dict(LAW, M4=LAW["M4"] + 1))
    with pytest.raises(titan.TitanError):
        gpu.set_ray_law(dict(LAW, M0=LAW["M0"] + 1, M4=LAW["M4"] - 1))
    gpu.set_ray_law(None)
    gpu.go(1)
    gpu.close()
