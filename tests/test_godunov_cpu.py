"""The oracle's restatement of the exact Godunov solver of HP faces
(Phys_param::Godunov_Solver_Alexashov, TITAN/source/Phys_param.cpp:1938-2385)
against the reference's own compiled solver: the golden vectors in
tests/golden/godunov_golden.npz (made by tests/golden/make_godunov_golden.py)
cover the four wave patterns, both pressure orders and the contact flag."""
import os

import numpy as np

import oracle_lib as ol

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "godunov_golden.npz")


def pattern(q1, q2, nrm, gamma=5.0 / 3.0):
    """Which of the reference's four wave patterns a case falls in (after its
    pressure-order swap): 'vacuum', 'two_rarefactions', 'shock_rarefaction', 'two_shocks'."""
    enI, enII = q1[1:4] @ nrm, q2[1:4] @ nrm
    pI, pII, rI, rII = q1[4], q2[4], q1[0], q2[0]
    if pI > pII:
        enI, enII, pI, pII, rI, rII = -enII, -enI, pII, pI, rII, rI
    g1, g2, gm = gamma - 1, gamma + 1, (gamma - 1) / gamma / 2
    cI, cII = np.sqrt(gamma * pI / rI), np.sqrt(gamma * pII / rII)
    a = np.sqrt(rI * (g2 * pII + g1 * pI) / 2)
    Uud, Urz, Uvk = (pII - pI) / a, -2 * cII / g1 * (1 - (pI / pII) ** gm), -2 * (cII + cI) / g1
    Udf = enI - enII
    if Udf < Uvk:
        return "vacuum"
    if Udf <= Urz:
        return "two_rarefactions"
    if Udf <= Uud:
        return "shock_rarefaction"
    return "two_shocks"


def test_golden_cases_cover_every_wave_pattern():
    g = np.load(GOLD)
    kinds = {pattern(g["q1"][i], g["q2"][i], g["nrm"][i]) for i in range(len(g["w"]))}
    assert kinds == {"vacuum", "two_rarefactions", "shock_rarefaction", "two_shocks"}
    assert (g["q1"][:, 4] > g["q2"][:, 4]).any() and (g["q1"][:, 4] < g["q2"][:, 4]).any()
    assert g["contact"].any()


def test_oracle_matches_reference_golden_bitwise(oracle_lib):
    g = np.load(GOLD)
    for i in range(len(g["w"])):
        out, ds, rc = ol.godunov("oracle", g["nrm"][i], g["w"][i], g["q1"][i], g["q2"][i], contact=g["contact"][i])
        assert rc == 0
        assert np.array_equal(out, g["flux"][i]), (i, out, g["flux"][i])
        assert np.array_equal(ds, g["ds"][i]), i


def test_oracle_matches_compiled_reference_on_fresh_cases(oracle_lib):
    if not os.path.exists(ol.REF_SO):
        import pytest
        pytest.skip("the reference solver is built only where the reference tree is present")
    nrm, w, q1, q2 = ol.random_godunov_cases(400, seed=99)
    for i in range(400):
        a = ol.godunov("oracle", nrm[i], w[i], q1[i], q2[i], contact=i % 3 == 0)
        b = ol.godunov("ref", nrm[i], w[i], q1[i], q2[i], contact=i % 3 == 0)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), i


def test_uniform_state_gives_the_physical_flux(oracle_lib):
    n = np.array([0.6, 0.0, 0.8])
    q = np.array([1.3, 0.4, -0.2, 0.1, 0.9])
    out, ds, rc = ol.godunov("oracle", n, 0.0, q, q)
    vn = q[1:4] @ n
    e = q[4] / (2.0 / 3.0) + 0.5 * q[0] * (q[1:4] @ q[1:4])
    want = np.concatenate([[q[0] * vn], q[0] * vn * q[1:4] + q[4] * n, [vn * (e + q[4])]])
    np.testing.assert_allclose(out, want, rtol=1e-12, atol=1e-14)
