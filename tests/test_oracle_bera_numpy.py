"""The oracle's Bera charge-exchange sources (oracle_sources) against a second,
separate restatement in numpy, written from the reference's text:

* the zone of a cell, Setka::determ_zone (TITAN/source/Setka_physics.cpp:1427-1460):
  1 or 2 (Zone_1 or not) where Q / rho < 50, else 4 or 3 (Zone_4 or not);
* the thermal protons, Phys_param::Plasma_components_1 (Phys_param.cpp:628-665),
  called with zone - 1 (Setka_physics.cpp:769, 777), with the floors of :796-801;
* the neutral fluids' temperatures, 2 p / max(rho, 1e-9) (:817-822);
* the rates U_bera, Um_bera, UE_bera (:746-764) and sigma = (1 - a2 ln U)^2 (:860-861);
* the momentum and energy exchange terms Hm, HE (:913-928) and the plasma's sums
  (:988-1000), scaled by n_H / Kn (:1236-1240).

Two transcriptions that agree to rounding on seeded cells of every zone pin the
oracle's restatement of this part of the step beyond its invariants; the
thermal-proton split is also pinned bit for bit to the reference's compiled
code, live where the reference tree is built and through a golden file it
generated everywhere."""
import ctypes

import numpy as np
import pytest

import oracle_lib as ol

ME_DMP = 1.0 / 1836.15


def _sources_numpy(st, H, ctype, a2, nH_lism, Kn):
    """[4, n] m_x, m_y, m_z, E of the plasma, written from the reference text."""
    rho, vx, vy, vz, p, Q, rho_He = st[0], st[1], st[2], st[3], st[4], st[8], st[9]
    zone = np.where(Q / rho < 50.0, np.where(ctype == 1, 1, 2), np.where(ctype == 4, 4, 3))
    zone_ = zone - 1
    al = np.where(zone_ <= 2, 2.0, 1.0)
    rho_p = -(ME_DMP * al * rho_He + 4.0 * (-rho + rho_He)) / (4.0 * (1.0 + ME_DMP))
    T_p = 8.0 * (1.0 + ME_DMP) * p / (8.0 * rho - (7.0 - al + (-1.0 + al) * ME_DMP) * rho_He)
    rho_p = np.where(rho_p <= 1e-8, 1e-8, rho_p)
    T_p = np.where(T_p <= 1e-8, 1e-8, T_p)
    T_p = np.where(T_p > 1e5, 1e5, T_p)
    Vp = np.stack([vx, vy, vz])
    S = np.zeros((4, st.shape[1]))
    pi = np.pi
    nh = H.shape[0] // 5
    for k in range(nh):
        rho_h = H[5 * k]
        Vh = H[5 * k + 1:5 * k + 4]
        T_h = 2.0 * H[5 * k + 4] / np.maximum(rho_h, 1e-9)

        def norm(a):
            return np.sqrt((a[0] * a[0] + a[1] * a[1]) + a[2] * a[2])

        def dot(a, b):
            return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]

        def U(T1, T2, V1, V2):
            uu = norm(V1 - V2)
            return np.sqrt((4.0 / pi) * (T1 + T2) + uu * uu)

        def Um(T1, T2, V1, V2):
            uu = norm(V1 - V2)
            return np.sqrt((16.0 / pi) * T1 + (9.0 * pi / 4.0) * T2 + 4.0 * (uu * uu))

        def UE(T1, T2, V1, V2):
            uu = norm(V1 - V2)
            return np.sqrt((4.0 / pi) * T1 + (64.0 / 9.0 / pi) * T2 + uu * uu)

        U_ph, U_hp = U(T_p, T_h, Vp, Vh), U(T_h, T_p, Vh, Vp)
        Um_ph, Um_hp = Um(T_p, T_h, Vp, Vh), Um(T_h, T_p, Vh, Vp)
        UE_ph, UE_hp = UE(T_p, T_h, Vp, Vh), UE(T_h, T_p, Vh, Vp)
        sig_ph = (1.0 - a2 * np.log(U_ph)) ** 2
        sig_hp = (1.0 - a2 * np.log(U_hp)) ** 2
        dV = Vp - Vh
        # Hm[H + p] (neutral -> proton) and Hm[p + H] (proton -> neutral), :913-918
        Hm_hp = sig_hp * rho_p * rho_h * (U_hp * Vp + T_p / Um_hp * dV)
        Hm_ph = sig_ph * rho_p * rho_h * (U_ph * Vh - T_h / Um_ph * dV)
        # HE, :920-926
        HE_hp = sig_hp * rho_p * rho_h * (0.5 * U_hp * dot(Vp, Vp) + T_p / Um_hp * dot(Vp, dV) +
                                          3.0 / 4.0 * T_p * UE_hp)
        HE_ph = sig_ph * rho_p * rho_h * (0.5 * U_ph * dot(Vh, Vh) - T_h / Um_ph * dot(Vh, dV) +
                                          3.0 / 4.0 * T_h * UE_ph)
        S[0:3] += -Hm_hp + Hm_ph
        S[3] += -HE_hp + HE_ph
    return S * (nH_lism / Kn)


def test_bera_sources_agree_with_a_second_restatement(titan, oracle_lib):
    rng = np.random.default_rng(11)
    n, nh = 4000, 4
    st = np.zeros((10, n))
    st[0] = 0.01 + 2.0 * rng.random(n)
    st[1:4] = 2.0 * rng.standard_normal((3, n))
    st[4] = 1e-3 + rng.random(n)
    st[5:8] = 0.3 * rng.standard_normal((3, n))
    st[8] = st[0] * np.where(rng.random(n) < 0.5, 10.0, 100.0)   # both sides of Q / rho = 50
    st[9] = st[0] * 0.1 * rng.random(n)
    H = np.zeros((5 * nh, n))
    for k in range(nh):
        H[5 * k] = 0.01 + 0.3 * rng.random(n)
        H[5 * k + 1:5 * k + 4] = 2.0 * rng.standard_normal((3, n))
        H[5 * k + 4] = 1e-3 + 0.2 * rng.random(n)
    ctype = rng.integers(0, 5, n).astype(np.int8)
    a2, nH_lism, Kn = 0.1307, 0.18, 0.4326
    m = ol.OMesh()
    m.ncell = n
    m.cell_type = ctype.ctypes.data_as(ctypes.POINTER(ctypes.c_int8))
    p = ol.OParams()
    p.gamma, p.par_a_2, p.par_n_H_LISM, p.par_Kn, p.nh = 5.0 / 3.0, a2, nH_lism, Kn, nh
    S_o = np.zeros((n, 4))
    L = ol.oracle()
    L.oracle_sources.argtypes = [ctypes.POINTER(ol.OMesh), ctypes.POINTER(ol.OParams), ol.D, ol.D, ol.D]
    st_c, H_c = np.ascontiguousarray(st), np.ascontiguousarray(H)
    L.oracle_sources(ctypes.byref(m), ctypes.byref(p), ol._p(st_c), ol._p(H_c), ol._p(S_o))
    S_n = _sources_numpy(st, H, ctype.astype(np.int64), a2, nH_lism, Kn)
    for k in range(4):
        scale = np.abs(S_n[k]).max()
        assert np.abs(S_o[:, k] - S_n[k]).max() <= 1e-12 * scale, k


@pytest.mark.skipif(not ol.ref_available(), reason="reference solver not built (no reference tree)")
def test_thermal_protons_match_the_compiled_reference(oracle_lib):
    """rho_Th and T_Th of the restatement above (and of the oracle, which agrees
    with it) against the reference's own compiled Phys_param::Plasma_components_1
    (Phys_param.cpp:628-665), for the 0-based zones 0-3 it is called with."""
    rng = np.random.default_rng(3)
    L = ol.ref()
    out = np.zeros(3)
    for zone_ in range(4):
        al = 2.0 if zone_ <= 2 else 1.0
        for _ in range(200):
            rho = 0.01 + 2.0 * rng.random()
            p = 1e-3 + rng.random()
            rho_He = rho * 0.2 * rng.random()
            L.titan_ref_plasma_components_1(zone_, rho, p, rho_He, ol._p(out))
            rho_p = -(ME_DMP * al * rho_He + 4.0 * (-rho + rho_He)) / (4.0 * (1.0 + ME_DMP))
            T_p = 8.0 * (1.0 + ME_DMP) * p / (8.0 * rho - (7.0 - al + (-1.0 + al) * ME_DMP) * rho_He)
            assert out[0] == rho_p and out[2] == T_p


def test_thermal_protons_match_the_reference_golden():
    """The same split against tests/golden/plasma_components_golden.npz, made
    by the compiled reference (make_plasma_golden.py): rho_Th, p_Th and T_Th
    bit for bit over zones 0-3, helium-rich cells included. Needs no reference
    tree."""
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "plasma_components_golden.npz"))
    rho, p, rho_He = g["rho"], g["p"], g["rho_he"]
    al = np.where(g["zone"] <= 2, 2.0, 1.0)
    rho_p = -(ME_DMP * al * rho_He + 4.0 * (-rho + rho_He)) / (4.0 * (1.0 + ME_DMP))
    p_p = p * (4.0 * rho - (4.0 + al * ME_DMP) * rho_He) / (8.0 * rho + (-7.0 + al + (1.0 - al) * ME_DMP) * rho_He)
    T_p = 8.0 * (1.0 + ME_DMP) * p / (8.0 * rho - (7.0 - al + (-1.0 + al) * ME_DMP) * rho_He)
    assert len(rho) == 1600 and np.any(g["out"][:, 0] <= 0.0)
    np.testing.assert_array_equal(g["out"][:, 0], rho_p)
    np.testing.assert_array_equal(g["out"][:, 1], p_p)
    np.testing.assert_array_equal(g["out"][:, 2], T_p)
