"""The closure's CPU side: the network oracle's gradient against finite
differences, and the feature / target / source mappings (csrc/closure.h
mirrored in titan_c-_b200/closure.py) as exact round trips."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mlp_oracle as mo  # noqa: E402


def _net(seed=0, n=64):
    rng = np.random.default_rng(seed)
    from importlib import import_module

    cl = import_module("titan_c-_b200.closure")
    p = cl.init_params(seed).astype(np.float64)
    p += 0.01 * rng.standard_normal(p.size) * (p != 0)
    X = rng.standard_normal((n, 8))
    norm = np.concatenate([np.zeros(8), np.ones(8), np.ones(5)])
    T = rng.standard_normal((n, 5))
    return p, norm, X, T


def test_parameter_layout_matches_the_header():
    txt = open(os.path.join(ROOT, "include", "titan_b200.h")).read()
    assert f"#define TITAN_MLP_NPARAM {mo.NPARAM}" in txt


def test_oracle_gradient_matches_finite_differences():
    p, norm, X, T = _net()
    w = np.array([1.0, 0.5, 2.0, 1.0, 0.25])
    loss, g = mo.loss_grad(p, norm, X, T, w, emulate_bf16=False)
    rng = np.random.default_rng(1)
    live = np.nonzero(p != 0)[0]
    live = np.concatenate([live, [o[1] for o in mo.offsets()]])  # biases too
    for i in rng.choice(live, 40, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mo.loss_grad(pp, norm, X, T, w, False)[0] - mo.loss_grad(pm, norm, X, T, w, False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-7, (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -3.140625, 0.0])
    assert list(mo.bf16(x)) == [1.0, 1.0, 1.0 + 2 ** -6, 1.0, -3.140625, 0.0]


def _plasma(titan, n=500, seed=3):
    rng = np.random.default_rng(seed)
    cc = rng.uniform(-50, 50, (3, n))
    st = np.zeros((10, n))
    st[0] = np.exp(rng.normal(-2, 1, n))
    st[1:4] = rng.normal(0, 2, (3, n))
    st[4] = np.exp(rng.normal(-3, 1, n))
    return st, cc


def test_frame_is_orthonormal_and_e1_follows_the_flow(titan):
    st, cc = _plasma(titan)
    st[1:4, :3] = 0.0                      # at rest: radial frame
    st[1:4, 3] = (-1.5, 0.0, 0.0)          # flow along the inflow axis
    e1, e2, e3 = titan.closure.frame(st, cc)
    for a in (e1, e2, e3):
        assert np.allclose(np.linalg.norm(a, axis=1), 1.0)
    assert np.allclose((e1 * e2).sum(1), 0.0, atol=1e-12)
    assert np.allclose((e1 * e3).sum(1), 0.0, atol=1e-12)
    V = st[1:4].T
    vm = np.linalg.norm(V, axis=1)
    assert np.allclose(e1[3:], V[3:] / vm[3:, None])
    assert np.allclose(e1[:3], (cc[:, :3] / np.linalg.norm(cc[:, :3], axis=0)).T)


def test_sources_invert_targets(titan):
    st, cc = _plasma(titan)
    rng = np.random.default_rng(5)
    mc = rng.standard_normal((5, st.shape[1]))
    mc[0] = np.abs(mc[0])
    T = titan.closure.targets(st, cc, mc, 0.18, 4.0)
    back = titan.closure.sources(st, cc, T, 0.18, 4.0)
    assert np.allclose(back, mc, rtol=1e-12, atol=1e-12)


def test_features_are_finite_and_proxy_is_bounded(titan):
    st, cc = _plasma(titan)
    X = titan.closure.features(st, cc, 0.18, 4.0)
    assert X.dtype == np.float32 and X.shape == (st.shape[1], 8)
    assert np.isfinite(X).all()
    assert (X[:, 7] <= np.log(0.18) + 1e-6).all() and (X[:, 7] >= np.log(0.18) - 30 - 1e-6).all()
    assert (np.abs(X[:, 6]) <= 1.0 + 1e-6).all()
