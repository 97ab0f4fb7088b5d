"""The oracle's cell update against a second, separate restatement in numpy,
written from the reference's text (TITAN/source/Setka_physics.cpp):

* the flux gather, POTOK[name] += sign * P<name> over the cell's faces in its
  own order, sign -1 where the cell is the face's cells[1] (:1671-1733);
* the conservative update of rho, Q, rho_He (rho_He floored at 0), velocity
  with the Powell term and the momentum source, B, and the pressure from the
  total energy with the energy source and the 8 pi literal (:1779-1902);
* the rho < 1e-7 reset to rho = 0.1 with the old velocity and B and p = rho / 2;
* the Zone_2 magnetic dissipation with tau = 1 (:1904-1917);
* the pressure floor p < 1e-8 -> 1e-6, rho_He > rho -> 0.1 rho, and B frozen
  where is_TVD is false (:1969-2028).

It is fed the oracle's own face fluxes and Bera sources of the step (those
have their own pins), on a stationary shell with zones, passive scalars and
neutral fluids, over a state pushed to trigger both floors in some cells. The
two must agree to rounding: an expression-order slip in either shows."""
import ctypes

import numpy as np

import oracle_lib as ol

C8PI = 25.13274122871834590768


def _cell_update_numpy(st, F, cell_faces, face_cells, S, vol, dt, gamma, ctype, tvd):
    nc = st.shape[1]
    g1 = gamma - 1.0
    cpi4 = 4.0 * np.pi
    PO = np.zeros((11, nc))
    for s in range(6):
        f = cell_faces[:, s]
        sign = np.where(face_cells[f, 0] == np.arange(nc), 1.0, -1.0)
        PO += sign[None, :] * F[f].T
    rho, vx, vy, vz, p = st[0], st[1], st[2], st[3], st[4]
    bx, by, bz, Q, rho_He = st[5], st[6], st[7], st[8], st[9]
    V = V2 = vol
    dsk = vx * bx + vy * by + vz * bz
    rho3 = rho * V / V2 - dt * PO[0] / V2
    null = rho3 < 1e-7
    rho3 = np.where(null, 0.1, rho3)
    Q3 = Q * V / V2 - dt * PO[9] / V2
    rho_He3 = rho_He * V / V2 - dt * PO[10] / V2
    rho_He3 = np.where(rho_He3 < 0.0, 0.0, rho_He3)
    u3 = (rho * vx * V / V2 - dt * (PO[1] + (bx / cpi4) * PO[8]) / V2 + dt * S[0]) / rho3
    v3 = (rho * vy * V / V2 - dt * (PO[2] + (by / cpi4) * PO[8]) / V2 + dt * S[1]) / rho3
    w3 = (rho * vz * V / V2 - dt * (PO[3] + (bz / cpi4) * PO[8]) / V2 + dt * S[2]) / rho3
    bx3 = bx * V / V2 - dt * (PO[5] + vx * PO[8]) / V2
    by3 = by * V / V2 - dt * (PO[6] + vy * PO[8]) / V2
    bz3 = bz * V / V2 - dt * (PO[7] + vz * PO[8]) / V2
    p3 = (((p / g1 + 0.5 * rho * (vx * vx + vy * vy + vz * vz) + (bx * bx + by * by + bz * bz) / C8PI) * V / V2
           - dt * (PO[4] + (dsk / cpi4) * PO[8]) / V2 + dt * S[3]) -
          0.5 * rho3 * (u3 * u3 + v3 * v3 + w3 * w3) - (bx3 * bx3 + by3 * by3 + bz3 * bz3) / C8PI) * g1
    z2 = ctype == 2
    tau = 1.0
    p4 = p3 + (dt / tau - (dt / tau) ** 2) * g1 * (bx3 * bx3 + by3 * by3 + bz3 * bz3) / (4.0 * np.pi)
    bx3, by3, bz3, p3 = (np.where(z2, bx3 - dt * bx3 / tau, bx3), np.where(z2, by3 - dt * by3 / tau, by3),
                         np.where(z2, bz3 - dt * bz3 / tau, bz3), np.where(z2, p4, p3))
    u3, v3, w3 = np.where(null, vx, u3), np.where(null, vy, v3), np.where(null, vz, w3)
    bx3, by3, bz3 = np.where(null, bx, bx3), np.where(null, by, by3), np.where(null, bz, bz3)
    p3 = np.where(null, rho3 / 2.0, p3)
    p3 = np.where(p3 < 1e-8, 1e-6, p3)
    rho_He3 = np.where(rho_He3 > rho3, rho3 * 0.1, rho_He3)
    keep = tvd == 0
    return np.stack([rho3, u3, v3, w3, p3, np.where(keep, bx, bx3), np.where(keep, by, by3),
                     np.where(keep, bz, bz3), Q3, rho_He3])


def test_cell_update_agrees_with_a_second_restatement(titan, oracle_lib):
    m, p, st, hf = titan.problems.heliosphere_shell(nq=6, nlayer=8, move=False, zones=True, npassive=2, nh=2)
    st = np.ascontiguousarray(st.copy())
    rng = np.random.default_rng(5)
    C = st.shape[1]
    st[9] = 0.05 * st[0]
    # toward the floors: scattered cells at a very low pressure, and three radial
    # layers of thin gas in a diverging flow (v = 5 x, div v > 0), whose middle
    # layer loses its mass within the step
    st[4, rng.choice(C, 20, replace=False)] = 1e-12
    lay = m["node_layer"][m["cell_nodes"]].min(axis=1)
    thin = (lay >= 3) & (lay <= 5)
    st[0, thin] = 1e-7
    st[4, thin] = 1e-9
    st[1:4, thin] = 5.0 * m["node_xyz"][m["cell_nodes"]].mean(axis=1)[thin].T
    run = ol.OracleRun(m, p)
    run.hf = np.ascontiguousarray(hf)
    dt = 0.05
    F, _, err = run.face_fluxes(st, dt)
    assert err == 0
    S_cell = np.zeros((C, 4))
    L = ol.oracle()
    L.oracle_sources.argtypes = [ctypes.POINTER(ol.OMesh), ctypes.POINTER(ol.OParams), ol.D, ol.D, ol.D]
    L.oracle_sources(ctypes.byref(run.mesh), ctypes.byref(run.params), ol._p(st), ol._p(run.hf), ol._p(S_cell))
    vol = run.geometry()["cell_volume"]
    want = _cell_update_numpy(st, F, m["cell_faces"], m["face_cells"], S_cell.T, vol, dt, p["gamma"],
                              m["cell_type"], m["cell_tvd"])
    got = st.copy()
    run.clock[:] = (dt, 0.0)
    info = run.go(got, 1)
    assert info.err_code == 0
    assert info.n_p_floor > 0 and info.n_rho_floor > 0    # both floors ran
    assert np.any(m["cell_type"] == 2) and np.any(m["cell_tvd"] == 0)
    for k in range(10):
        scale = np.abs(want[k]).max()
        assert np.abs(got[k] - want[k]).max() <= 1e-12 * scale, k
