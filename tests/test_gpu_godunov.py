"""The exact gas-dynamic Godunov solver of HP faces on the GPU
(Phys_param::Godunov_Solver_Alexashov, TITAN/source/Phys_param.cpp:1938-2385):
the batch entry against the reference's own solver (golden vectors from
tests/golden/make_godunov_golden.py), and whole steps with HP faces and
bn_in_p_on_HP against the oracle. The solver's Newton and bisection steps call
pow, where CUDA's math library and glibc may differ by an ulp; everything
else is the reference's arithmetic, so the bar is 1e-12 relative."""
import os

import numpy as np
import pytest

import oracle_lib as ol
from test_gpu_parity import REL, rel_err

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "godunov_golden.npz")


@pytest.fixture(scope="module")
def T(titan, built_lib):
    return titan


def batch(T, nrm, w, q1, q2, contact, gamma=5.0 / 3.0):
    N = T.native
    n = len(w)
    flux, ds = np.empty((n, 5)), np.empty((n, 3))
    rc = np.empty(n, dtype=np.int32)
    c = np.ascontiguousarray(contact, dtype=np.int8)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (nrm, w, q1, q2)]
    N.check(N.lib().titan_godunov_batch(n, N.ptr(arrs[0]), N.ptr(arrs[1]), N.ptr(arrs[2]), N.ptr(arrs[3]),
                                        N.ptr(c, N.I8), gamma, N.ptr(flux), N.ptr(ds), N.ptr(rc, N.I32)))
    return flux, ds, rc


def test_batch_matches_reference_golden(T):
    g = np.load(GOLD)
    flux, ds, rc = batch(T, g["nrm"], g["w"], g["q1"], g["q2"], g["contact"])
    assert (rc == 0).all()
    scale = np.maximum(np.abs(g["flux"]).max(axis=1, keepdims=True), 1e-300)
    assert (np.abs(flux - g["flux"]) / scale).max() <= REL
    assert (np.abs(ds - g["ds"]) / np.maximum(np.abs(g["ds"]).max(axis=1, keepdims=True), 1e-300)).max() <= REL
    exact = np.all(flux == g["flux"], axis=1).mean()
    assert exact > 0.5, exact       # most cases round identically; pow may differ by an ulp


def _hp_shell(T, move, zones, npassive):
    m, p, st, _ = T.problems.heliosphere_shell(nq=8, nlayer=8, move=move, zones=zones, npassive=npassive)
    layer = m["node_layer"]
    fn = m["face_nodes"]
    hp = np.all(layer[fn] == 4, axis=1)       # the radial faces of one spherical layer
    assert hp.sum() == 6 * 8 * 8
    m["face_surf"] = np.where(hp, 2, m["face_surf"]).astype(np.int8)
    p = dict(p, bn_in_p_on_hp=1)
    return m, p, st


@pytest.mark.parametrize("features", [dict(move=False, zones=False, npassive=0),
                                      dict(move=True, zones=True, npassive=2)])
def test_steps_with_hp_faces_match_oracle(T, oracle_lib, features):
    m, p, st = _hp_shell(T, **features)
    gpu = T.PlasmaStep(m, p)
    run = ol.OracleRun(m, p)
    gpu.upload_state(st)
    ns = 8 + p["npassive"]
    worst = 0.0
    for _ in range(10):
        before = np.ascontiguousarray(gpu.download_state())
        run.xyz[:] = gpu.nodes()
        run.clock[:] = (gpu.dt, gpu.t)
        gpu.go(1)
        assert run.go(before, 1).err_code == 0
        worst = max(worst, rel_err(gpu.download_state()[:ns], before[:ns]))
    assert worst <= REL, worst
    # the HP faces carry no magnetic or divB flux
    fl = gpu.face_fluxes()
    hp = m["face_surf"] == 2
    assert not fl[hp][:, 5:9].any()
    gpu.close()


def test_mixed_precision_step_with_hp_faces_runs(T):
    m, p, st = _hp_shell(T, move=True, zones=True, npassive=0)
    g = T.PlasmaStep(m, dict(p, flux_precision=32))
    g.upload_state(st)
    info = g.go(20)
    assert info["steps_done"] == 20
    assert np.isfinite(g.download_state()).all()
    g.close()
