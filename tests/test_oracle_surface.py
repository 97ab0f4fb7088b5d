"""The oracle's surface-tracking node motion (Setka::Culc_Velocity_surface,
TITAN/source/Setka_move.cpp:111-1358, and Luch::dvigenie, Luch.cpp:6-739)
pinned by construction on the CPU:

* with every surface held still the step equals the step on a mesh whose
  nodes do not move, up to rounding (the rays place their nodes again from
  the segment rule every step, as Luch::dvigenie does);
* in a uniform flow every face's contact speed is the flow's normal speed, so
  each HP node moves by dt times velocity_HP times the mean of (u . n) n over
  its faces, projected on its radial direction — formed here in numpy from
  the oracle's own face normals;
* the other nodes of each ray stay on the ray, in order, at their initial
  fraction of the segment between the surface nodes and the ray's ends;
* null_bn_on_HP leaves the cells next to the HP without normal B."""
import numpy as np
import pytest

import oracle_lib as ol


def _shell(titan, nq=6, nlayer=10):
    m, p, st, _ = titan.problems.heliosphere_shell(nq=nq, nlayer=nlayer, move=True)
    m["node_amp"] = np.zeros(m["node_xyz"].shape[0])
    m["node_phase"] = np.zeros(m["node_xyz"].shape[0])
    return m, p, st


SURF = dict(velocity_TS=1.0, velocity_HP=1.0, velocity_BS=1.0, move_TS=1, move_HP=1, move_BS=1, null_bn_on_HP=0)


def test_still_surfaces_give_the_fixed_mesh_step(titan, oracle_lib):
    m, p, st = _shell(titan)
    for layer, kind in ((4, 1), (6, 2), (8, 3)):
        titan.mesh.mark_shell_surface(m, layer, kind)
    rays = titan.mesh.shell_rays(m)
    still = dict(SURF, move_TS=0, move_HP=0, move_BS=0)
    a, b = np.ascontiguousarray(st.copy()), np.ascontiguousarray(st.copy())
    ra = ol.OracleRun(m, p, surface=still, rays=rays)
    rb = ol.OracleRun(m, p)            # prescribed motion with zero amplitude
    x0 = ra.xyz.copy()
    assert ra.go(a, 5).err_code == 0
    assert rb.go(b, 5).err_code == 0
    assert np.abs(ra.xyz - x0).max() <= 1e-15 * np.abs(x0).max()
    for k in range(8):
        assert np.abs(a[k] - b[k]).max() <= 1e-11 * np.abs(b[k]).max(), k


def _uniform(m, u=(0.3, -0.2, 0.1), B=(0.05, 0.0, 0.1)):
    C = m["cell_nodes"].shape[0]
    st = np.zeros((10, C))
    st[0], st[4] = 1.0, 1.0
    st[1:4] = np.asarray(u)[:, None]
    st[5:8] = np.asarray(B)[:, None]
    return st


def test_hp_nodes_move_with_the_contact_speed_of_a_uniform_flow(titan, oracle_lib):
    m, p, _ = _shell(titan)
    titan.mesh.mark_shell_surface(m, 5, 2)
    rays = titan.mesh.shell_rays(m)
    u = np.array([0.3, -0.2, 0.1])
    st = np.ascontiguousarray(_uniform(m, u))
    vel = 0.7
    run = ol.OracleRun(m, p, surface=dict(SURF, velocity_HP=vel, move_TS=0, move_BS=0), rays=rays)
    x0 = run.xyz.copy()
    fn = run.geometry()["face_normal"]
    dt = run.clock[0]
    assert run.go(st, 1).err_code == 0
    x1 = run.xyz
    # numpy: mean over each HP node's faces of vel (u . n) n, projected on x/|x|
    hp = np.nonzero(m["face_surf"] == 2)[0]
    V = np.zeros_like(x0)
    cnt = np.zeros(len(x0))
    for f in hp:
        for i in m["face_nodes"][f]:
            V[i] += vel * (fn[f] @ u) * fn[f]
            cnt[i] += 1
    moved = cnt > 0
    V[moved] /= cnt[moved, None]
    B = x0[moved] / np.linalg.norm(x0[moved], axis=1, keepdims=True)
    expect = x0[moved] + (np.sum(V[moved] * B, axis=1) * dt)[:, None] * B
    np.testing.assert_allclose(x1[moved], expect, rtol=0, atol=1e-13 * np.abs(x0).max())
    assert np.abs(x1[moved] - x0[moved]).max() > 1e-9 * dt * 1e5   # they did move


def test_ray_nodes_keep_their_segment_fractions(titan, oracle_lib):
    m, p, st = _shell(titan)
    for layer, kind in ((4, 1), (6, 2), (8, 3)):
        titan.mesh.mark_shell_surface(m, layer, kind)
    rays = titan.mesh.shell_rays(m)
    run = ol.OracleRun(m, p, surface=dict(SURF, velocity_TS=50.0, velocity_HP=50.0, velocity_BS=50.0), rays=rays)
    x0 = run.xyz.copy()
    s = np.ascontiguousarray(st.copy())
    assert run.go(s, 3).err_code == 0
    x1 = run.xyz
    r0 = np.linalg.norm(x0[rays], axis=2)
    r1 = np.linalg.norm(x1[rays], axis=2)
    anchors = [0, 4, 6, 8, rays.shape[1] - 1]
    assert np.abs(r1[:, [4, 6, 8]] - r0[:, [4, 6, 8]]).max() > 0     # the surfaces moved
    assert np.array_equal(x1[rays[:, 0]], x0[rays[:, 0]])              # the ends did not
    assert np.array_equal(x1[rays[:, -1]], x0[rays[:, -1]])
    assert (np.diff(r1, axis=1) > 0).all()                             # order kept
    d = x0[rays[:, 0]] / np.linalg.norm(x0[rays[:, 0]], axis=1, keepdims=True)
    for a, b in zip(anchors[:-1], anchors[1:]):
        for j in range(a + 1, b):
            f0 = (r0[:, j] - r0[:, a]) / (r0[:, b] - r0[:, a])
            f1 = (r1[:, j] - r1[:, a]) / (r1[:, b] - r1[:, a])
            np.testing.assert_allclose(f1, f0, rtol=0, atol=1e-12)
            cross = np.cross(x1[rays[:, j]], d)
            assert np.abs(cross).max() <= 1e-12 * r1[:, j].max()


def test_null_bn_on_hp_removes_the_normal_field_of_the_hp_cells(titan, oracle_lib):
    m, p, _ = _shell(titan)
    titan.mesh.mark_shell_surface(m, 5, 2)
    rays = titan.mesh.shell_rays(m)
    st = np.ascontiguousarray(_uniform(m, B=(0.3, -0.1, 0.2)))
    run = ol.OracleRun(m, p, surface=dict(SURF, move_TS=0, move_BS=0, null_bn_on_HP=1), rays=rays)
    fn = run.geometry()["face_normal"]
    # after one step the HP cells' B . n is far below that of the same step
    # without null_bn_on_HP (the step's own fluxes change B only a little)
    ref = np.ascontiguousarray(st.copy())
    run2 = ol.OracleRun(m, p, surface=dict(SURF, move_TS=0, move_BS=0, null_bn_on_HP=0), rays=rays)
    assert run.go(st, 1).err_code == 0
    assert run2.go(ref, 1).err_code == 0
    hp = np.nonzero(m["face_surf"] == 2)[0]
    cells = m["face_cells"][hp]
    bn_null = np.abs(np.einsum("ij,ij->i", st[5:8, cells[:, 0]].T, fn[hp]))
    bn_ref = np.abs(np.einsum("ij,ij->i", ref[5:8, cells[:, 0]].T, fn[hp]))
    assert bn_null.mean() < 0.2 * bn_ref.mean(), (bn_null.mean(), bn_ref.mean())


def test_a_shorter_ray_ends_at_its_last_node(titan, oracle_lib):
    """Rays of different lengths: a ray padded with -1 treats its last node as
    its outer end; the node it leaves out stays where it is."""
    m, p, st = _shell(titan)
    for layer, kind in ((4, 1), (6, 2), (8, 3)):
        titan.mesh.mark_shell_surface(m, layer, kind)
    rays = titan.mesh.shell_rays(m)
    short = rays.copy()
    short[::2, -1] = -1
    run = ol.OracleRun(m, p, surface=dict(SURF, velocity_TS=50.0, velocity_HP=50.0, velocity_BS=50.0), rays=short)
    x0 = run.xyz.copy()
    s = np.ascontiguousarray(st.copy())
    assert run.go(s, 2).err_code == 0
    x1 = run.xyz
    assert np.array_equal(x1[rays[::2, -1]], x0[rays[::2, -1]])     # left out
    assert np.array_equal(x1[rays[::2, -2]], x0[rays[::2, -2]])     # the new outer end
    assert not np.array_equal(x1[rays[::2, -3]], x0[rays[::2, -3]])  # its BS node still moves


def _bumped_shell(titan, layer, kind, bump):
    """A shell with one surface and one of its nodes pushed outward by `bump` (relative)."""
    m, p, st = _shell(titan)
    titan.mesh.mark_shell_surface(m, layer, kind)
    node = int(np.nonzero(m["node_layer"] == layer)[0][17])
    m["node_xyz"] = m["node_xyz"].copy()
    m["node_xyz"][node] *= 1.0 + bump
    return m, p, st, node


def test_bs_smoothing_pulls_a_bumped_node_back(titan, oracle_lib):
    """sglag_BS (Setka_move.cpp:1136-1211): a BS node pushed out of the surface
    moves inward relative to the same step without smoothing, toward the mean
    of itself and its neighbours."""
    m, p, st, node = _bumped_shell(titan, 5, 3, 0.02)
    rays = titan.mesh.shell_rays(m)
    out = {}
    for on in (0, 1):
        run = ol.OracleRun(m, p, surface=dict(SURF, sglag_BS=on, sglag_BS_k=0.5), rays=rays)
        s = np.ascontiguousarray(st.copy())
        assert run.go(s, 1).err_code == 0
        out[on] = np.linalg.norm(run.xyz[node])
    assert out[1] < out[0], out


@pytest.mark.parametrize("layer,kind,key,vel", [(4, 1, "sglag_TS", "velocity_TS"), (6, 2, "sglag_HP", "velocity_HP")])
def test_sphere_smoothing_term_as_numpy_forms_it(titan, oracle_lib, layer, kind, key, vel):
    """sglag_TS / sglag_HP (Setka_move.cpp:454-558, 559-620): the node's mean
    velocity takes one more term, v_s = velocity_X k (B2 - x) / dt with
    B2 = c + (mean |x_j - c| / |x - c|) (x - c), c the sphere centre fitted at
    set-up; the node's radial displacement is then (n_f d_off + dt v_s . x/|x|)
    / (n_f + 1), n_f its surface faces, d_off the displacement without it. The
    reference's fit passes the sphere through the origin (it solves
    2 p . c = |p|^2), so on an origin-centred surface the term points outward."""
    m, p, st, node = _bumped_shell(titan, layer, kind, 0.02)
    rays = titan.mesh.shell_rays(m)
    k_sph, velo = 0.5, 1.0
    d, runs = {}, {}
    for on in (0, 1):
        run = ol.OracleRun(m, p, surface=dict(SURF, **{key: on, key + "_k_sphere": k_sph, vel: velo}), rays=rays)
        x0 = run.xyz.copy()
        dt = run.clock[0]
        s = np.ascontiguousarray(st.copy())
        assert run.go(s, 1).err_code == 0
        d[on] = np.linalg.norm(run.xyz[node]) - np.linalg.norm(x0[node])
        runs[on] = run
    c = np.zeros((m["node_xyz"].shape[0], 3))
    import ctypes
    ol.oracle().oracle_surface_centres(ctypes.byref(runs[1].mesh), ol._p(np.ascontiguousarray(x0)), ol._p(c))
    faces = np.nonzero((m["face_surf"] == kind) & np.any(m["face_nodes"] == node, axis=1))[0]
    nbs = np.setdiff1d(np.unique(m["face_nodes"][faces]), [node])
    A, C = x0[node], c[node]
    r = np.mean(np.linalg.norm(x0[nbs] - C, axis=1))
    B2 = C + (r / np.linalg.norm(A - C)) * (A - C)
    v_s = velo * k_sph * (B2 - A) / dt
    nf = len(faces)
    expect = (nf * d[0] + dt * (v_s @ (A / np.linalg.norm(A)))) / (nf + 1)
    assert abs(d[1] - expect) <= 1e-9 * abs(expect), (d, expect)


def test_smoothing_off_changes_nothing(titan, oracle_lib):
    """All smoothing flags off: the same step as before smoothing existed, bit for bit."""
    m, p, st = _shell(titan)
    for layer, kind in ((4, 1), (6, 2), (8, 3)):
        titan.mesh.mark_shell_surface(m, layer, kind)
    rays = titan.mesh.shell_rays(m)
    res = []
    for extra in ({}, dict(sglag_TS=0, sglag_HP=0, sglag_BS=0, sglag_TS_k_sphere=0.3, sglag_BS_k=0.3)):
        run = ol.OracleRun(m, p, surface=dict(SURF, **extra), rays=rays)
        s = np.ascontiguousarray(st.copy())
        assert run.go(s, 2).err_code == 0
        res.append((s, run.xyz.copy()))
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])


# The A_Luch spacing law (Luch::dvigenie, TITAN/source/Luch.cpp:9-152): node
# counts and radii of Geo_param; a ray of M0 + M1 + M2 + M3 + M4 + 5 = 24 nodes.
LAW = dict(M0=2, M1=4, M11=1, M2=5, M3=4, M4=4, R0=1.0, R1=2.0, R5=100.0,
           da1=1.2, da2=0.8, da3=0.9, da4=1.1, da5=0.5)
LAW_SLOTS = (7, 13, 18)   # TS, HP, BS


def law_shell(titan, nq=6, R=(10.0, 20.0, 40.0), **kw):
    """A shell whose layers sit where the A_Luch law puts them, with the
    TS, HP and BS surfaces on the law's slots."""
    radii = titan.mesh.a_luch_radii(LAW, *R)
    m, p, st, hf = titan.problems.heliosphere_shell(nq=nq, nlayer=len(radii) - 1, move=True, radii=radii, **kw)
    for slot, kind in zip(LAW_SLOTS, (1, 2, 3)):
        titan.mesh.mark_shell_surface(m, slot, kind)
    return m, p, st, titan.mesh.shell_rays(m)


def test_a_luch_law_is_a_fixed_point_of_still_surfaces(titan, oracle_lib):
    m, p, st, rays = law_shell(titan)
    still = dict(SURF, move_TS=0, move_HP=0, move_BS=0)
    run = ol.OracleRun(m, p, surface=still, rays=rays, ray_law=LAW)
    x0 = run.xyz.copy()
    assert run.go(np.ascontiguousarray(st.copy()), 3).err_code == 0
    assert np.abs(run.xyz - x0).max() <= 1e-13 * np.abs(x0).max()


def test_a_luch_law_places_ray_nodes_from_the_moved_surfaces(titan, oracle_lib):
    """After steps that move the three surfaces, every ray's radii are the
    law's radii for its current TS, HP and BS radii (mesh.a_luch_radii, a
    separate numpy restatement), on the ray's own direction."""
    m, p, st, rays = law_shell(titan)
    surf = dict(SURF, velocity_TS=30.0, velocity_HP=30.0, velocity_BS=30.0)
    run = ol.OracleRun(m, p, surface=surf, rays=rays, ray_law=LAW)
    x0 = run.xyz.copy()
    s = np.ascontiguousarray(st.copy())
    assert run.go(s, 4).err_code == 0
    r = np.linalg.norm(run.xyz[rays], axis=2)
    moved = np.abs(r[:, list(LAW_SLOTS)] - np.linalg.norm(x0[rays][:, list(LAW_SLOTS)], axis=2))
    assert moved.max() > 1e-6
    for k in range(rays.shape[0]):
        want = titan.mesh.a_luch_radii(LAW, *r[k, list(LAW_SLOTS)])
        assert np.abs(r[k] - want).max() <= 1e-12 * want.max(), k
    # every node of a ray on the ray's initial direction
    d0 = x0[rays[:, 0]] / np.linalg.norm(x0[rays[:, 0]], axis=1)[:, None]
    u = run.xyz[rays] / r[:, :, None]
    assert np.abs(u - d0[:, None, :]).max() <= 1e-12


def test_hp_tail_nodes_move_across_the_axis_only(titan, oracle_lib):
    """With hp_tail (Setka_move.cpp:1237-1247) an HP node with x < 0 moves
    along (0, y, z): its x stays, its distance from the x axis changes; HP
    nodes with x >= 0 still move along their own direction."""
    m, p, st = _shell(titan)
    titan.mesh.mark_shell_surface(m, 6, 2)
    rays = titan.mesh.shell_rays(m)
    surf = dict(SURF, move_TS=0, move_BS=0, hp_tail=1)
    run = ol.OracleRun(m, p, surface=surf, rays=rays)
    x0 = run.xyz.copy()
    assert run.go(np.ascontiguousarray(st.copy()), 2).err_code == 0
    hp = rays[:, 6]
    tail = x0[hp, 0] < 0
    assert tail.any() and (~tail).any()
    assert np.array_equal(run.xyz[hp[tail], 0], x0[hp[tail], 0])
    assert np.abs(np.hypot(run.xyz[hp[tail], 1], run.xyz[hp[tail], 2]) -
                  np.hypot(x0[hp[tail], 1], x0[hp[tail], 2])).max() > 0
    head = hp[~tail]
    u0 = x0[head] / np.linalg.norm(x0[head], axis=1)[:, None]
    u1 = run.xyz[head] / np.linalg.norm(run.xyz[head], axis=1)[:, None]
    assert np.abs(u1 - u0).max() < 1e-12
