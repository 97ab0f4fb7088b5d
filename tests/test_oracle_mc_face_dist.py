"""The oracle's Monte-Carlo launch from a tabulated face distribution (the
reference's face AMR functions as input: AMR_f::Culk_SpotokV and
Get_random_velosity, TITAN/source/AMR_f.cpp:4-96, AMR_cell::
Get_random_velosity_in_cell, AMR_cell.cpp:273-326), pinned on the CPU by
construction with one table face and no other inflow:

* the pass's inflow is the face's sum over leaves of box volume * f * |box
  centre x| times the face area;
* without charge exchange a neutral keeps its start velocity, so every
  neutral's velocity, in the face's frame, lies inside one of its leaves;
* the leaves are hit in proportion to their weights, and within a leaf the
  normal component follows the flux-weighted law x = sqrt(xL^2 + r (xR^2 -
  xL^2)) (its mean is 2 (xR^3 - xL^3) / (3 (xR^2 - xL^2))).

And the outgoing tallies (AMR_f::Add_particle, Normir_velocity_volume):
every neutral stopped on a tallied face is accounted for in its leaves and
moments.
"""
import numpy as np

import oracle_lib as ol

MC = dict(n_H=0.18, u_H=(-2.6, 0.0, 0.0), cp_H=1.3)


def _frame(n):
    a = np.array([1.0, 0.0, 0.0]) if abs(n[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    t = np.cross(n, a)
    t /= np.linalg.norm(t)
    return np.concatenate([n, t, np.cross(n, t)])


def test_single_table_face_launch(titan, oracle_lib):
    m, p, st, _ = titan.problems.heliosphere_shell(nq=6, nlayer=6, move=False)
    p = dict(p, par_Kn=1e30)                     # no charge exchange
    geo = ol.OracleRun(m, p).geometry()
    f = int(np.nonzero(m["face_type"] == 2)[0][0])
    E = _frame(-geo["face_normal"][f])           # Vn into the cell (the normal points out)
    # three leaves of different sizes and values, one split finer in x
    box = np.array([[0.0, 1.0, -2.0, 2.0, -2.0, 2.0],
                    [1.0, 1.5, -2.0, 0.0, -1.0, 1.0],
                    [1.5, 4.0, 0.5, 1.5, -3.0, -1.0]])
    fv = np.array([0.2, 1.0, 0.35])
    fd = dict(face=[f], side=[0], frame=E[None, :], leaf_ptr=[0, 3], leaf_box=box, leaf_f=fv)
    n = 60000
    _, trace, total, lost = ol.mc_pass(m, st, p, n_particles=n, seed=3, face_types=0, face_dist=fd, **MC)
    assert lost == 0
    V = (box[:, 1] - box[:, 0]) * (box[:, 3] - box[:, 2]) * (box[:, 5] - box[:, 4])
    w = V * fv * np.abs((box[:, 0] + box[:, 1]) / 2.0)
    assert abs(total - w.sum() * geo["face_area"][f]) <= 1e-12 * total
    v = trace[:, 3:6]
    loc = np.stack([v @ E[0:3], v @ E[3:6], v @ E[6:9]], axis=1)
    inside = np.stack([(loc[:, 0] >= b[0] - 1e-12) & (loc[:, 0] <= b[1] + 1e-12) &
                       (loc[:, 1] >= b[2] - 1e-12) & (loc[:, 1] <= b[3] + 1e-12) &
                       (loc[:, 2] >= b[4] - 1e-12) & (loc[:, 2] <= b[5] + 1e-12) for b in box], axis=1)
    assert np.all(inside.sum(axis=1) >= 1)
    leaf = np.argmax(inside, axis=1)             # the leaves do not overlap
    share = np.bincount(leaf, minlength=3) / n
    assert np.abs(share - w / w.sum()).max() < 0.01
    for k, b in enumerate(box):
        xs = loc[leaf == k, 0]
        mean = 2.0 * (b[1] ** 3 - b[0] ** 3) / (3.0 * (b[1] ** 2 - b[0] ** 2))
        assert abs(xs.mean() - mean) < 0.02 * (b[1] - b[0]) + 4.0 * xs.std() / np.sqrt(len(xs))


def test_outgoing_tallies_account_for_every_stopped_neutral(titan, oracle_lib):
    """Tallies (AMR_f::Add_particle and Normir_velocity_volume, AMR_f.cpp:240-336)
    on an interior sphere of faces: per face, the normalised leaves give back
    the stopped weight (sum of f * box volume * area * box-centre x = Smu *
    area), and the faces together hold mu times the neutrals whose trace ends
    with kind 3 (stopped on a tallied face)."""
    m, p, st, _ = titan.problems.heliosphere_shell(nq=6, nlayer=8, move=False)
    p = dict(p, par_Kn=3.0)
    geo = ol.OracleRun(m, p).geometry()
    on = np.all(m["node_layer"][m["face_nodes"]] == 5, axis=1) & (m["face_cells"][:, 1] >= 0)
    faces = np.nonzero(on)[0]
    cc = m["node_xyz"][m["cell_nodes"]].mean(axis=1)
    fc = m["face_cells"][faces]
    side = (np.linalg.norm(cc[fc[:, 1]], axis=1) > np.linalg.norm(cc[fc[:, 0]], axis=1)).astype(np.int8)
    frame = np.array([_frame(geo["face_normal"][f] * (1.0 if s == 0 else -1.0)) for f, s in zip(faces, side)])
    xe, ye = np.linspace(0.0, 8.0, 5), np.linspace(-6.0, 6.0, 4)
    i, j, k = [a.ravel() for a in np.meshgrid(np.arange(4), np.arange(3), np.arange(3), indexing="ij")]
    b = np.stack([xe[i], xe[i + 1], ye[j], ye[j + 1], ye[k], ye[k + 1]], axis=1)
    ft = dict(face=faces, side=side, frame=frame, leaf_ptr=np.arange(len(faces) + 1) * len(b),
              leaf_box=np.tile(b, (len(faces), 1)))
    n = 40000
    _, trace, total, lost = ol.mc_pass(m, st, p, n_particles=n, seed=4, face_tally=ft, **MC)
    mu = total / n
    stopped = int(np.sum(trace[:, 7] % 4 == 3))
    assert stopped > 0 and ft["unplaced"] == 0
    area = geo["face_area"][faces]
    V = (b[:, 1] - b[:, 0]) * (b[:, 3] - b[:, 2]) * (b[:, 5] - b[:, 4])
    cx = (b[:, 0] + b[:, 1]) / 2.0
    f = ft["leaf_f"].reshape(len(faces), len(b))
    per_face = (f * V[None, :] * cx[None, :]).sum(axis=1) * area
    smu = ft["moments"][:, 1] * area
    assert np.allclose(per_face, smu, rtol=1e-12, atol=1e-12 * smu.max())
    assert abs(smu.sum() - mu * stopped) <= 1e-9 * mu * stopped
