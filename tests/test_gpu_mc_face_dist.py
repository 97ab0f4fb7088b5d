"""Monte-Carlo neutrals launched from tabulated face distributions
(titan_set_mc_face_dist: the reference's face AMR functions as input,
TITAN/source/Setka_MK.cpp:1225-1575, AMR_f.cpp:4-96, AMR_cell.cpp:273-326).

* Neutral by neutral against the oracle's restatement (oracle_mc_pass with the
  same tables): irregular leaf boxes on outer boundary faces and on a layer of
  interior faces, entering either side; the inflow total to 1e-12 and nearly
  every neutral's end record to 1e-9 (the tracer's FMA contraction and CUDA's
  libm can part a history at a threshold, as in test_gpu_mc_oracle.py).
* Tables that discretise the drifting Maxwellian on every inflow face give the
  analytic launch's velocity moments: without charge exchange a neutral's end
  velocity is its start velocity, so the mean velocity and mean speed squared
  of the two launches agree within sampling and discretisation error.
* Outgoing tallies (titan_set_mc_face_tally: AMR_f::Add_particle and
  Normir_velocity_volume, AMR_f.cpp:240-336) on an interior sphere of faces
  against the oracle's restatement, and the zone coupling they make with the
  tabulated launch: a second pass launched from the first pass's tallies
  reproduces the inner zone's neutral content of one uncoupled pass.
* Bad tables and tallies are refused before anything runs.
"""
import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu

MC = dict(n_H=0.18, u_H=(-2.6, 0.0, 0.0), cp_H=1.3)


def _frame(n):
    """Vn = n and two unit vectors across it."""
    a = np.array([1.0, 0.0, 0.0]) if abs(n[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    t = np.cross(n, a)
    t /= np.linalg.norm(t)
    return np.concatenate([n, t, np.cross(n, t)])


def _maxwell(w, u, cp, nH):
    return nH / (np.pi ** 1.5 * cp ** 3) * np.exp(-np.sum((w - u) ** 2, axis=-1) / cp ** 2)


def _tables(g, m, faces, sides, grid, irregular, seed=0):
    """Tables for `faces` (original ids): the frame from the face normal
    toward the entered cell; leaves on a grid of local velocities in x-major
    order, f the drifting Maxwellian in local coordinates (irregular: an
    extra x edge inside the first column and random factors on f)."""
    rng = np.random.default_rng(seed)
    nrm = g.geometry()["face_normal"]
    u = np.asarray(MC["u_H"])
    cp, nH = MC["cp_H"], MC["n_H"]
    nx, ny = grid
    frame, ptr, box, fv = [], [0], [], []
    for f, sd in zip(faces, sides):
        E = _frame(nrm[f] * (1.0 if sd else -1.0))
        frame.append(E)
        ul = np.array([u @ E[0:3], u @ E[3:6], u @ E[6:9]])
        xe = np.linspace(0.0, max(ul[0], 0.0) + 5.0 * cp, nx + 1)
        if irregular:
            xe = np.insert(xe, 1, 0.5 * xe[1])
        ye = np.linspace(ul[1] - 5.0 * cp, ul[1] + 5.0 * cp, ny + 1)
        ze = np.linspace(ul[2] - 5.0 * cp, ul[2] + 5.0 * cp, ny + 1)
        i, j, k = np.meshgrid(np.arange(len(xe) - 1), np.arange(ny), np.arange(ny), indexing="ij")
        i, j, k = i.ravel(), j.ravel(), k.ravel()
        b = np.stack([xe[i], xe[i + 1], ye[j], ye[j + 1], ze[k], ze[k + 1]], axis=1)
        c = np.stack([(b[:, 0] + b[:, 1]) / 2, (b[:, 2] + b[:, 3]) / 2, (b[:, 4] + b[:, 5]) / 2], axis=1)
        val = _maxwell(c, ul, cp, nH)
        if irregular:
            val = val * (0.5 + rng.random(len(val)))
        box.append(b)
        fv.append(val)
        ptr.append(ptr[-1] + len(val))
    return dict(face=np.asarray(faces, np.int32), side=np.asarray(sides, np.int8), frame=np.array(frame),
                leaf_ptr=np.asarray(ptr, np.int64), leaf_box=np.concatenate(box), leaf_f=np.concatenate(fv))


def _shell(titan):
    m, p, st, _ = titan.problems.heliosphere_shell(nq=8, nlayer=12, move=False)
    return m, p, st


def test_face_tables_match_oracle_neutral_by_neutral(titan, oracle_lib):
    m, p, st = _shell(titan)
    p = dict(p, par_Kn=2.0)
    g = titan.PlasmaStep(m, p)
    g.upload_state(st)
    outer = np.nonzero(m["face_type"] == 2)[0][::2]
    # interior spherical faces of node layer 6 (all four nodes on it)
    on6 = np.all(m["node_layer"][m["face_nodes"]] == 6, axis=1)
    inner_layer = np.nonzero(on6 & (m["face_cells"][:, 1] >= 0))[0][:64]
    assert len(inner_layer) == 64
    faces = np.concatenate([outer, inner_layer])
    sides = np.concatenate([np.zeros(len(outer), int), np.arange(len(inner_layer)) % 2])
    fd = _tables(g, m, faces, sides, grid=(4, 3), irregular=True)
    g.set_mc_face_dist(fd)
    n = 40000
    trace = np.zeros((n, 8))
    out, info = g.mc_sources(n_particles=n, seed=5, trace=trace, **MC)
    c_n2o, f_n2o, n_n2o = g.permutation()
    g.close()
    mr, c_o2n = ol.renumbered_mesh(m, c_n2o, f_n2o, n_n2o)
    f_o2n = np.empty_like(f_n2o)
    f_o2n[f_n2o] = np.arange(len(f_n2o))
    fdo = dict(fd, face=f_o2n[fd["face"]])
    tal, otr, total, lost = ol.mc_pass(mr, st[:, c_n2o], p, n_particles=n, seed=5, face_dist=fdo, **MC)
    assert abs(info["inflow_rate"] - total) <= 1e-12 * total
    same = (trace[:, 6] == otr[:, 6]) & (trace[:, 7] == otr[:, 7])
    close = np.all(np.abs(trace[:, :6] - otr[:, :6]) <= 1e-9 * (1.0 + np.abs(otr[:, :6])), axis=1)
    assert (same & close).mean() >= 0.99, (same & close).mean()
    tal_o = tal[:, c_o2n]
    for k in range(5):
        scale = np.abs(tal_o[k]).max()
        assert (np.abs(out[k] - tal_o[k]) <= 1e-9 * scale).mean() >= 0.9, k


def test_maxwellian_tables_reproduce_the_analytic_launch(titan):
    m, p, st = _shell(titan)
    p = dict(p, par_Kn=1e30)   # no charge exchange: end velocity = start velocity
    g = titan.PlasmaStep(m, p)
    g.upload_state(st)
    n = 200000
    t0 = np.zeros((n, 8))
    _, info0 = g.mc_sources(n_particles=n, seed=9, trace=t0, face_types=1 << 2, **MC)
    faces = np.nonzero(m["face_type"] == 2)[0]
    fd = _tables(g, m, faces, np.zeros(len(faces), int), grid=(16, 20), irregular=False)
    g.set_mc_face_dist(fd)
    t1 = np.zeros((n, 8))
    _, info1 = g.mc_sources(n_particles=n, seed=9, trace=t1, face_types=1 << 2, **MC)
    g.set_mc_face_dist(None)
    _, info2 = g.mc_sources(n_particles=n, seed=9, face_types=1 << 2, **MC)
    g.close()
    assert info2["inflow_rate"] == info0["inflow_rate"]
    # the tables carry the Maxwellian's inflow to the grid's accuracy
    assert abs(info1["inflow_rate"] / info0["inflow_rate"] - 1.0) < 0.02
    for t in (t0, t1):
        assert np.all(t[:, 6] == 0)          # no exchanges
    v0, v1 = t0[:, 3:6], t1[:, 3:6]
    cp = MC["cp_H"]
    assert np.abs(v1.mean(axis=0) - v0.mean(axis=0)).max() < 0.03 * cp
    s0, s1 = (v0 ** 2).sum(axis=1).mean(), (v1 ** 2).sum(axis=1).mean()
    assert abs(s1 / s0 - 1.0) < 0.03


def test_bad_face_tables_are_refused(titan):
    m, p, st = _shell(titan)
    g = titan.PlasmaStep(m, p)
    bnd = np.nonzero(m["face_cells"][:, 1] < 0)[0][:2]
    good = _tables(g, m, bnd, [0, 0], grid=(2, 2), irregular=False)
    g.set_mc_face_dist(good)
    for bad in (dict(good, side=np.array([1, 0], np.int8)),                       # side 1 of a boundary face
                dict(good, face=np.array([bnd[0], bnd[0]], np.int32)),             # a face twice
                dict(good, leaf_ptr=np.array([0, 5000, len(good["leaf_f"])])),     # leaves out of order
                dict(good, leaf_box=good["leaf_box"] * np.array([-1, 1, 1, 1, 1, 1.0])),  # xL < 0 or xR < xL
                dict(good, leaf_f=np.zeros_like(good["leaf_f"]))):                 # lets nothing in
        with pytest.raises(titan.TitanError):
            g.set_mc_face_dist(bad)
    g.set_mc_face_dist(None)
    g.close()


def _sphere_faces(m, layer=9):
    """The interior faces of node layer `layer`, the side of each face's
    outer cell, and the unit vector from that cell through the face."""
    on = np.all(m["node_layer"][m["face_nodes"]] == layer, axis=1) & (m["face_cells"][:, 1] >= 0)
    faces = np.nonzero(on)[0]
    cc = m["node_xyz"][m["cell_nodes"]].mean(axis=1)
    fc = m["face_cells"][faces]
    r0, r1 = np.linalg.norm(cc[fc[:, 0]], axis=1), np.linalg.norm(cc[fc[:, 1]], axis=1)
    side = (r1 > r0).astype(np.int8)           # the outer cell's side
    return faces, side


def _tally_tables(g, faces, side, nx, ny, xmax=8.0, ymax=6.0):
    """Leaf grids for faces, frame Vn pointing out of the side cell."""
    nrm = g.geometry()["face_normal"]
    xe = np.linspace(0.0, xmax, nx + 1)
    ye = np.linspace(-ymax, ymax, ny + 1)
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(ny), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    b = np.stack([xe[i], xe[i + 1], ye[j], ye[j + 1], ye[k], ye[k + 1]], axis=1)
    frame = np.array([_frame(nrm[f] * (1.0 if s == 0 else -1.0)) for f, s in zip(faces, side)])
    return dict(face=faces.astype(np.int32), side=side.astype(np.int8), frame=frame,
                leaf_ptr=np.arange(len(faces) + 1, dtype=np.int64) * len(b),
                leaf_box=np.tile(b, (len(faces), 1)))


def test_face_tallies_match_oracle(titan, oracle_lib):
    m, p, st = _shell(titan)
    p = dict(p, par_Kn=2.0)
    g = titan.PlasmaStep(m, p)
    g.upload_state(st)
    faces, side = _sphere_faces(m)
    ft = _tally_tables(g, faces, side, 4, 4)
    g.set_mc_face_tally(ft)
    n = 40000
    trace = np.zeros((n, 8))
    g.mc_sources(n_particles=n, seed=7, trace=trace, **MC)
    got = g.mc_face_tally()
    c_n2o, f_n2o, n_n2o = g.permutation()
    g.close()
    mr, c_o2n = ol.renumbered_mesh(m, c_n2o, f_n2o, n_n2o)
    f_o2n = np.empty_like(f_n2o)
    f_o2n[f_n2o] = np.arange(len(f_n2o))
    fto = dict(ft, face=f_o2n[ft["face"]])
    ol.mc_pass(mr, st[:, c_n2o], p, n_particles=n, seed=7, face_tally=fto, **MC)
    kinds = trace[:, 7] % 4
    assert (kinds == 3).mean() > 0.03              # many neutrals stopped on the sphere
    assert got["unplaced"] == fto["unplaced"]
    for a, b in ((got["leaf_f"], fto["leaf_f"]), (got["moments"], fto["moments"])):
        scale = np.abs(b).max()
        assert (np.abs(a - b) <= 1e-9 * scale).mean() >= 0.9
        assert abs(a.sum() - b.sum()) <= 0.05 * np.abs(b).sum()


def test_zone_coupling_through_face_tables(titan):
    """Zone A (the whole mesh, neutrals stopped when they cross the layer-9
    sphere inward) tallies its outgoing tables; zone B (launched only from
    those tables, into the inner cells) then carries the neutrals on. Without
    charge exchange a straight path crosses the sphere inward at most once, so
    the inner zone's neutral content of B equals that of one pass with no
    tallies, up to sampling and the tables' velocity resolution."""
    m, p, st = _shell(titan)
    p = dict(p, par_Kn=1e30)
    g = titan.PlasmaStep(m, p)
    g.upload_state(st)
    cc = m["node_xyz"][m["cell_nodes"]].mean(axis=1)
    rsph = np.linalg.norm(m["node_xyz"][m["node_layer"] == 9], axis=1).mean()
    inner = np.linalg.norm(cc, axis=1) < rsph
    geo = g.geometry()
    vol, area = geo["cell_volume"], geo["face_area"]
    n = 4000000
    full, _ = g.mc_sources(n_particles=n, seed=21, face_types=1 << 2, **MC)
    faces, side = _sphere_faces(m)
    ft = _tally_tables(g, faces, side, 10, 12, xmax=8.0, ymax=6.0)
    g.set_mc_face_tally(ft)
    _, infoA = g.mc_sources(n_particles=n, seed=22, face_types=1 << 2, **MC)
    tal = g.mc_face_tally()
    g.set_mc_face_tally(None)
    keep = np.zeros(len(faces), bool)
    lp = ft["leaf_ptr"]
    for i in range(len(faces)):
        keep[i] = tal["leaf_f"][lp[i]:lp[i + 1]].sum() > 0
    sel = np.nonzero(keep)[0]
    nl = lp[1] - lp[0]
    fd = dict(face=faces[sel], side=(1 - side[sel]).astype(np.int8), frame=ft["frame"][sel],
              leaf_ptr=np.arange(len(sel) + 1, dtype=np.int64) * nl,
              leaf_box=np.concatenate([ft["leaf_box"][lp[i]:lp[i + 1]] for i in sel]),
              leaf_f=np.concatenate([tal["leaf_f"][lp[i]:lp[i + 1]] for i in sel]))
    g.set_mc_face_dist(fd)
    zoneB, infoB = g.mc_sources(n_particles=n, seed=23, face_types=0, **MC)
    g.close()
    # B's inflow is what A stopped on the sphere: sum of Smu times face area
    assert tal["unplaced"] == 0
    crossed = float((tal["moments"][:, 1] * area[faces]).sum())
    assert abs(infoB["inflow_rate"] / crossed - 1.0) < 1e-9
    content_full = float((full[0] * vol)[inner].sum())
    content_B = float((zoneB[0] * vol)[inner].sum())
    assert abs(content_B / content_full - 1.0) < 0.05, (content_B, content_full)


def test_bad_face_tallies_are_refused(titan):
    m, p, st = _shell(titan)
    g = titan.PlasmaStep(m, p)
    g.upload_state(st)
    faces, side = _sphere_faces(m)
    ft = _tally_tables(g, faces[:3], side[:3], 2, 2)
    bnd = np.nonzero(m["face_cells"][:, 1] < 0)[0][:3]
    with pytest.raises(titan.TitanError):
        g.set_mc_face_tally(dict(ft, face=bnd.astype(np.int32), side=np.ones(3, np.int8)))
    with pytest.raises(titan.TitanError):
        g.set_mc_face_tally(dict(ft, leaf_box=ft["leaf_box"] * np.array([1, -1, 1, 1, 1, 1.0])))
    g.set_mc_face_tally(ft)
    with pytest.raises(titan.TitanError):
        g.mc_face_tally()                      # no pass since the tallies were set
    g.mc_sources(n_particles=1000, seed=1, **MC)
    assert g.mc_face_tally()["leaf_f"].shape == (len(ft["leaf_box"]),)
    g.close()
