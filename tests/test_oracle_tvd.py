"""The oracle's second-order (TVD) reconstruction, Setka_gran_snos.cpp:188-735,
with the neighbours of Setka::Init_TVD (Setka_physics.cpp:646-738): properties
that hold by construction, checked on the CPU.

* On a regular cube every interior face's second-order neighbours are the
  cells one step further along the face normal, except next to the boundary.
* A uniform state reconstructs to itself (zero slopes), so the second-order
  face fluxes equal the first-order ones.
* A linear profile on a regular mesh reconstructs exactly at the face (the two
  one-sided slopes agree, minmod returns them).
* On an all-Zone_1 shell, a radial wind with rho r^2, p r^(2 gamma), |V|
  and B_r r^2 constant reconstructs exactly at the face through the
  spherical-component branch.
"""
import numpy as np
import pytest

import oracle_lib as ol


def _run(titan, m, **over):
    p = titan.problems.params(tvd=1, **over)
    return ol.OracleRun(m, p), p


def test_cube_neighbours_lie_along_the_normal(titan, oracle_lib):
    m = titan.mesh.cube_mesh(6)
    run, _ = _run(titan, m)
    g = run.geometry()
    cc, fn = g["cell_center"], g["face_normal"]
    fc = m["face_cells"]
    h = 1.0 / 6
    interior = np.nonzero(fc[:, 1] >= 0)[0]
    tvd = run.face_tvd
    assert (tvd[fc[:, 1] < 0, 1] == -1).all()
    for f in interior:
        A, B = fc[f]
        for side, (cel, sgn) in enumerate([(A, -1.0), (B, 1.0)]):
            want = cc[cel] + sgn * h * fn[f]
            nb = tvd[f, side]
            inside = np.all((want > 0) & (want < 1))
            if inside:
                assert nb >= 0
                np.testing.assert_allclose(cc[nb], want, atol=1e-12)
            else:
                assert nb == -1 or not np.allclose(cc[nb], want, atol=1e-9)


def test_uniform_state_gives_first_order_fluxes(titan, oracle_lib):
    m = titan.mesh.cube_mesh(6)
    C = m["cell_nodes"].shape[0]
    st = np.zeros((10, C))
    st[0], st[1], st[2], st[4], st[5], st[6] = 1.3, 0.2, -0.1, 0.7, 0.4, 0.9
    r2, _ = _run(titan, m)
    r1 = ol.OracleRun(m, titan.problems.params())
    f2, d2, e2 = r2.face_fluxes(np.ascontiguousarray(st))
    f1, d1, e1 = r1.face_fluxes(np.ascontiguousarray(st))
    assert e1 == e2 == 0
    np.testing.assert_array_equal(f2, f1)
    LR, used = r2.face_states(st)
    assert used.sum() > 0


def test_linear_profile_is_exact_at_the_face(titan, oracle_lib):
    m = titan.mesh.cube_mesh(8)
    run, _ = _run(titan, m)
    g = run.geometry()
    cc, fcen = g["cell_center"], g["face_center"]
    a = np.array([0.3, -0.2, 0.5])
    st = np.zeros((10, cc.shape[0]))
    st[0] = 2.0 + cc @ a
    st[4] = 1.0 + 0.5 * (cc @ a)
    st[1] = 0.1 + cc[:, 0]
    LR, used = run.face_states(st)
    # faces whose neighbours are collinear (next to the boundary Init_TVD may
    # pick a lateral cell, and the line then carries the lateral gradient)
    fc, tvd, fn = m["face_cells"], run.face_tvd, g["face_normal"]
    h = 1.0 / 8
    sel = used == 1
    for f in np.nonzero(sel)[0]:
        A, B = fc[f]
        sel[f] = (np.allclose(cc[tvd[f, 0]], cc[A] - h * fn[f], atol=1e-12)
                  and np.allclose(cc[tvd[f, 1]], cc[B] + h * fn[f], atol=1e-12))
    assert sel.sum() > 100
    exact_rho = 2.0 + fcen[sel] @ a
    np.testing.assert_allclose(LR[sel, 0, 0], exact_rho, rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(LR[sel, 1, 0], exact_rho, rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(LR[sel, 0, 1], 0.1 + fcen[sel, 0], rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("nq", [6, 9])
def test_radial_wind_is_exact_on_zone1(titan, oracle_lib, nq):
    m, p, _, _ = titan.problems.heliosphere_shell(nq=nq, nlayer=6, move=False)
    m["cell_type"] = np.ones_like(m["cell_type"])       # every cell Zone_1
    m["cell_tvd"] = np.ones_like(m["cell_tvd"])
    p = dict(p, tvd=1)
    run = ol.OracleRun(m, p)
    g = run.geometry()
    cc, fcen = g["cell_center"], g["face_center"]
    r = np.linalg.norm(cc, axis=1)
    rh = cc / r[:, None]
    gam = p["gamma"]
    st = np.zeros((10, cc.shape[0]))
    st[0] = 3.0 / r ** 2
    st[4] = 0.2 / r ** (2 * gam)
    st[1:4] = (1.7 * rh).T
    st[5:8] = (0.4 * rh / r[:, None] ** 2).T
    LR, used = run.face_states(st)
    sel = np.nonzero(used == 1)[0]
    assert len(sel) > 100
    rf = np.linalg.norm(fcen[sel], axis=1)
    gh = fcen[sel] / rf[:, None]
    for side in (0, 1):
        s = LR[sel, side]
        np.testing.assert_allclose(s[:, 0], 3.0 / rf ** 2, rtol=1e-11)
        np.testing.assert_allclose(s[:, 4], 0.2 / rf ** (2 * gam), rtol=1e-11)
        np.testing.assert_allclose(s[:, 1:4], 1.7 * gh, rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(s[:, 5:8], 0.4 * gh / rf[:, None] ** 2, rtol=1e-10, atol=1e-14)


def test_second_order_step_is_conservative(titan, oracle_lib):
    """Brio-Wu on the cube with second-order faces: the step's mass change is
    exactly the boundary outflow (interior faces cancel), the run stays finite,
    and it differs from the first-order run."""
    m, p, st, meth = titan.problems.brio_wu_cube(12)
    p = dict(p, tvd=1)
    run = ol.OracleRun(m, p)
    run.set_face_method(meth)
    s = np.ascontiguousarray(st.copy())
    run.go(s, 5)
    vol = run.geometry()["cell_volume"]
    dt = run.clock[0]
    fl, _, err = run.face_fluxes(s, time=dt)
    assert err == 0
    bnd = m["face_cells"][:, 1] < 0
    m0 = (s[0] * vol).sum()
    info = run.go(s, 1)
    assert info.err_code == 0 and np.isfinite(s).all()
    dm = (s[0] * vol).sum() - m0
    np.testing.assert_allclose(dm, -dt * fl[bnd, 0].sum(), rtol=1e-9, atol=1e-15)
    s1 = np.ascontiguousarray(st.copy())
    p1 = dict(p, tvd=0)
    r1 = ol.OracleRun(m, p1)
    r1.set_face_method(meth)
    r1.go(s1, 6)
    assert not np.array_equal(s, s1)
