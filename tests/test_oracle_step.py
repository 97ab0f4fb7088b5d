"""The oracle's step loop on CPU: invariants the reference's step has by construction."""
import numpy as np

import oracle_lib as ol


def _mass(run, st):
    return float(np.sum(st[0] * run.geometry()["cell_volume"]))


def test_uniform_flow_stays_uniform(titan, oracle_lib):
    m = titan.mesh.cube_mesh(6)
    p = titan.problems.params(soft_fixups=0)
    run = ol.OracleRun(m, p)
    run.set_face_method(np.full(m["face_nodes"].shape[0], 3))
    C = m["cell_nodes"].shape[0]
    st = np.zeros((10, C))
    st[0], st[1], st[2], st[3], st[4] = 1.3, 0.2, -0.1, 0.05, 0.7
    st[5], st[6], st[7] = 0.4, 0.3, -0.2
    st0 = st.copy()
    info = run.go(st, 5)
    assert info.err_code == 0 and info.steps_done == 5
    np.testing.assert_allclose(st[:8], st0[:8], rtol=1e-13, atol=1e-13)


def test_mass_changes_only_through_boundary(titan, oracle_lib):
    m, p, st, meth = titan.problems.brio_wu_cube(8)
    run = ol.OracleRun(m, p)
    run.set_face_method(meth)
    st = np.ascontiguousarray(st)
    # boundary flux of the first step (dt = 1e-5)
    fl, dtn, err = run.face_fluxes(st)
    assert err == 0
    bnd = m["face_cells"][:, 1] < 0
    m0 = _mass(run, st)
    run.go(st, 1)
    m1 = _mass(run, st)
    assert abs((m1 - m0) - (-1e-5 * fl[bnd, 0].sum())) <= 1e-13 * m0


def test_brio_wu_is_z_invariant_and_bounded(titan, oracle_lib):
    m, p, st, meth = titan.problems.brio_wu_cube(12)
    run = ol.OracleRun(m, p)
    run.set_face_method(meth)
    st = np.ascontiguousarray(st)
    info = run.go(st, 30)
    assert info.err_code == 0
    cc = m["node_xyz"][m["cell_nodes"]].mean(axis=1)
    k = np.round(cc[:, 2] * 12 - 0.5).astype(int)
    ij = np.round(cc[:, 0] * 12 - 0.5).astype(int) * 12 + np.round(cc[:, 1] * 12 - 0.5).astype(int)
    ref = np.zeros((12 * 12, 10))
    ref[ij[k == 0]] = st[:, k == 0].T
    np.testing.assert_allclose(st.T, ref[ij], rtol=1e-12, atol=1e-12)
    assert st[0].min() > 0.1 and st[0].max() < 1.05
    assert np.all(st[4] > 0)


def test_cfl_dt_is_applied_on_the_next_step(titan, oracle_lib):
    m, p, st, meth = titan.problems.brio_wu_cube(6)
    run = ol.OracleRun(m, p)
    run.set_face_method(meth)
    st = np.ascontiguousarray(st)
    fl, dtn, err = run.face_fluxes(st)
    run.go(st, 1)
    assert run.clock[0] == dtn     # the CFL minimum of step 1 becomes dt of step 2
    assert run.clock[1] == 1e-5    # step 1 used the initial 1e-5


def test_heliosphere_problem_steps_with_all_features(titan, oracle_lib):
    m, p, st, hf = titan.problems.heliosphere_shell(nq=4, nlayer=4, zones=True, npassive=2, nh=4)
    run = ol.OracleRun(m, p)
    run.hf = np.ascontiguousarray(hf)
    st = np.ascontiguousarray(st)
    x0 = run.xyz.copy()
    info = run.go(st, 3)
    assert info.err_code == 0, (info.err_code, info.err_index)
    assert np.all(np.isfinite(st))
    moved = np.linalg.norm(run.xyz - x0, axis=1).max()
    # |dx| <= amplitude * elapsed time for the prescribed radial motion
    assert 0 < moved <= 1e-3 * run.clock[1] * (1 + 1e-12)
