"""Learned charge-exchange closure: features, targets, training and use.

The network (csrc/closure_mlp.cu, csrc/closure_train.cu) maps a cell's plasma
state to the charge-exchange sources that the Monte-Carlo neutral solver
(PlasmaStep.mc_sources, after Setka::MK_fly_immit in
TITAN/source/Setka_MK.cpp:1752-2314) produces there, so the plasma loop can
run between Monte-Carlo passes without re-tracing neutrals.

Inputs (8): log rho, u_r, |u_t|, log(p/rho), log r, theta (the angle from
the upwind axis +x), the cosine of the angle between the plasma velocity and
the inflow direction -x, and the log of a cold-model neutral density
n_proxy = n_inf exp(-lambda theta / (r sin theta)). lambda = 0 (a flat proxy)
suits a generator with charge exchange only, which conserves the neutrals.
Outputs (5): n_H / n_proxy, then the plasma momentum source in the
frame (e1 = V/|V|, e2 = -x made orthogonal to e1, e3 = e1 x e2) and the energy
source, each divided by rho n_proxy; all five divided by a per-output scale
of the training set. The plasma mass source of charge exchange is zero
(Setka_physics.cpp:970), so the first output carries the neutral density.

Everything here mirrors csrc/closure.h (features, frame, proxy); training and
inference run on the GPU through the C ABI.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import native as N

NIN, NOUT, NPARAM = 8, 5, N.MLP_NPARAM
_LAYERS = [(16, 128), (128, 128), (128, 128), (128, 128), (128, 16)]


def log_proxy(cc: np.ndarray, n_inf: float, lam: float) -> np.ndarray:
    """log n_proxy per cell; cc [3][n] or [n][3]."""
    x, y, z = (cc if cc.shape[0] == 3 else cc.T)
    r = np.sqrt(x * x + y * y + z * z)
    th = np.arccos(np.clip(x / r, -1.0, 1.0))
    s = np.maximum(np.sin(th), 1e-3)
    return np.log(n_inf) + np.maximum(-lam * th / (r * s), -30.0)


def features(state: np.ndarray, cc: np.ndarray, n_inf: float, lam: float) -> np.ndarray:
    """X [n][8] float32 from the state [>=5][n] and the cell centres [3][n]."""
    rho, vx, vy, vz, p = state[:5]
    x, y, z = cc
    r = np.sqrt(x * x + y * y + z * z)
    ur = (vx * x + vy * y + vz * z) / r
    v2 = vx * vx + vy * vy + vz * vz
    vm = np.sqrt(v2)
    X = np.empty((rho.shape[0], NIN), dtype=np.float32)
    X[:, 0] = np.log(np.maximum(rho, 1e-30))
    X[:, 1] = ur
    # |u_t| = |v x r| / r: no cancellation for a nearly radial flow
    X[:, 2] = np.sqrt((vy * z - vz * y) ** 2 + (vz * x - vx * z) ** 2 + (vx * y - vy * x) ** 2) / r
    X[:, 3] = np.log(np.maximum(p / rho, 1e-30))
    X[:, 4] = np.log(r)
    X[:, 5] = np.arccos(np.clip(x / r, -1.0, 1.0))
    X[:, 6] = np.where(vm > 0.0, -vx / np.where(vm > 0.0, vm, 1.0), 0.0)
    X[:, 7] = log_proxy(cc, n_inf, lam)
    return X


def frame(state: np.ndarray, cc: np.ndarray):
    """(e1, e2, e3), each [n][3]: e1 = V/|V| (radial where V = 0), e2 = the
    inflow direction -x made orthogonal to e1, e3 = e1 x e2."""
    V = np.stack(state[1:4], axis=1)
    vm = np.linalg.norm(V, axis=1)
    rad = (cc / np.linalg.norm(cc, axis=0)).T
    e1 = np.where(vm[:, None] > 0.0, V / np.where(vm > 0.0, vm, 1.0)[:, None], rad)
    d = -e1[:, 0]
    e2 = -d[:, None] * e1
    e2[:, 0] -= 1.0
    n2 = np.linalg.norm(e2, axis=1)
    bad = n2 < 1e-12
    e2[bad] = (0.0, 1.0, 0.0)
    n2[bad] = 1.0
    e2 /= n2[:, None]
    return e1, e2, np.cross(e1, e2)


def targets(state, cc, mc: np.ndarray, n_inf: float, lam: float) -> np.ndarray:
    """Unscaled outputs T [n][5] from Monte-Carlo sources mc [5][n] (n_H, S_m, S_E)."""
    npx = np.exp(log_proxy(cc, n_inf, lam))
    norm = state[0] * npx
    e1, e2, e3 = frame(state, cc)
    S = mc[1:4].T
    T = np.empty((state.shape[1], NOUT))
    T[:, 0] = mc[0] / npx
    T[:, 1] = (S * e1).sum(1) / norm
    T[:, 2] = (S * e2).sum(1) / norm
    T[:, 3] = (S * e3).sum(1) / norm
    T[:, 4] = mc[4] / norm
    return T


def sources(state, cc, Y: np.ndarray, n_inf: float, lam: float) -> np.ndarray:
    """[5][n] (n_H, S_m, S_E) from unscaled outputs Y [n][5] (the inverse of targets)."""
    npx = np.exp(log_proxy(cc, n_inf, lam))
    norm = state[0] * npx
    e1, e2, e3 = frame(state, cc)
    out = np.empty((5, state.shape[1]))
    out[0] = Y[:, 0] * npx
    m = norm[:, None] * (Y[:, 1:2] * e1 + Y[:, 2:3] * e2 + Y[:, 3:4] * e3)
    out[1:4] = m.T
    out[4] = norm * Y[:, 4]
    return out


def init_params(seed: int = 0) -> np.ndarray:
    """He-scaled normal weights, zero biases, padding zero."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, dtype=np.float32)
    o = 0
    for li, (i, j) in enumerate(_LAYERS):
        W = rng.standard_normal((i, j)) * np.sqrt((2.0 if li < 4 else 1.0) / (NIN if li == 0 else i))
        if li == 0:
            W[NIN:] = 0.0
        if li == 4:
            W[:, NOUT:] = 0.0
        p[o:o + i * j] = W.ravel()
        o += i * j + j
    return p


def make_norm(X: np.ndarray, T: np.ndarray) -> np.ndarray:
    """norm [21] float32: feature mean [8], 1/std [8] (0 for a constant
    feature, which the network then ignores), output scale [5] (RMS of T)."""
    mean = X.astype(np.float64).mean(axis=0)
    std = X.astype(np.float64).std(axis=0)
    live = std > 1e-6 * (1.0 + np.abs(mean))
    istd = np.where(live, 1.0 / np.where(live, std, 1.0), 0.0)
    scale = np.sqrt((T * T).mean(axis=0))
    return np.concatenate([mean, istd, np.maximum(scale, 1e-30)]).astype(np.float32)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Closure:
    """A trained (or initial) network with its normalisation and proxy constants."""

    def __init__(self, n_inf: float, lam: float, params: np.ndarray | None = None,
                 norm: np.ndarray | None = None, seed: int = 0, envelope=None):
        self.n_inf, self.lam = float(n_inf), float(lam)
        self.params = _f32(init_params(seed) if params is None else params)
        self.norm = None if norm is None else _f32(norm)
        self.envelope = None if envelope is None else (_f32(envelope[0]), _f32(envelope[1]))
        self._lib = N.lib()

    @classmethod
    def load(cls, path: str) -> "Closure":
        """A network saved by train_closure.py (params, norm, proxy, training envelope)."""
        d = np.load(path)
        env = (d["envelope_lo"], d["envelope_hi"]) if "envelope_lo" in d else None
        return cls(float(d["n_inf"]), float(d["lam"]), d["params"], d["norm"], envelope=env)

    def set_fallback(self, step, mc_sources: np.ndarray | None) -> None:
        """Cells outside the training envelope take mc_sources[1:5] (a titan_mc_sources
        result, [5][ncell]) instead of the network; None keeps the previous table."""
        if self.envelope is None:
            raise ValueError("this closure has no training envelope")
        lo, hi = self.margined_envelope()
        src = None if mc_sources is None else np.ascontiguousarray(mc_sources[1:5], dtype=np.float64)
        N.check(self._lib.titan_set_closure_fallback(step.ctx, N.ptr(lo, N.F32), N.ptr(hi, N.F32), N.ptr(src)))

    def fallback_from_mc(self, step) -> None:
        """The fallback table from the step's last Monte-Carlo pass, on the device."""
        N.check(self._lib.titan_closure_fallback_from_mc(step.ctx))

    def margined_envelope(self, rel: float = 0.01):
        """The training envelope widened by `rel` of each feature's range plus
        1e-3 (1 + |bound|): the kernel forms features in FP32 with fast
        logarithms, and a feature that was constant in training (zero range,
        e.g. a flat proxy) must not push every cell outside."""
        lo = self.envelope[0].astype(np.float64)
        hi = self.envelope[1].astype(np.float64)
        w = hi - lo
        return (_f32(lo - rel * w - 1e-3 * (1.0 + np.abs(lo))), _f32(hi + rel * w + 1e-3 * (1.0 + np.abs(hi))))

    @staticmethod
    def outside(step) -> int:
        """Cells outside the training envelope in the last step."""
        v = ctypes.c_int64(0)
        N.check(N.lib().titan_closure_outside(step.ctx, ctypes.byref(v)))
        return int(v.value)

    # -- training -------------------------------------------------------------
    def fit(self, X: np.ndarray, T: np.ndarray, epochs: int = 20, batch: int = 4096, lr: float = 2e-3,
            lr_decay: float = 0.9, weights=None, row_weights=None, seed: int = 0) -> np.ndarray:
        """Adam on the GPU over (X, T unscaled); returns the mean loss per epoch.
        weights: per output [5]; row_weights: per row (scaled to mean 1), e.g.
        the cell volume, in proportion to which the Monte-Carlo samples a cell."""
        if self.norm is None:
            self.norm = make_norm(X, T)
        rng = np.random.default_rng(seed)
        order = rng.permutation(X.shape[0])
        Xs = _f32(X[order])
        Ts = _f32(T[order] / self.norm[2 * NIN:])
        w = _f32(np.ones(NOUT) if weights is None else weights)
        rw = None
        if row_weights is not None:
            rw = np.asarray(row_weights, dtype=np.float64)[order]
            rw = _f32(rw / rw.mean())
        o = N.TitanMlpTrainOpts(epochs=int(epochs), batch=int(batch), lr=lr, beta1=0.9, beta2=0.999,
                                lr_decay=lr_decay)
        losses = np.zeros(epochs, dtype=np.float32)
        N.check(self._lib.titan_mlp_train(N.ptr(self.params, N.F32), N.ptr(self.norm, N.F32), N.ptr(Xs, N.F32),
                                          N.ptr(Ts, N.F32), N.ptr(w, N.F32), N.ptr(rw, N.F32), Xs.shape[0],
                                          ctypes.byref(o), N.ptr(losses, N.F32)))
        return losses

    def grad(self, X, Tscaled, weights=None, row_weights=None):
        """(loss, grad [NPARAM], Y [n][5]) of one batch, scaled targets, on the GPU."""
        X, T = _f32(X), _f32(Tscaled)
        w = _f32(np.ones(NOUT) if weights is None else weights)
        rw = None if row_weights is None else _f32(row_weights)
        g = np.empty(NPARAM, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        Y = np.empty((X.shape[0], NOUT), dtype=np.float32)
        N.check(self._lib.titan_mlp_grad(N.ptr(self.params, N.F32), N.ptr(self.norm, N.F32), N.ptr(X, N.F32),
                                         N.ptr(T, N.F32), N.ptr(w, N.F32), N.ptr(rw, N.F32), X.shape[0],
                                         N.ptr(g, N.F32), N.ptr(loss, N.F32), N.ptr(Y, N.F32)))
        return float(loss[0]), g, Y

    # -- inference ------------------------------------------------------------
    def forward(self, X: np.ndarray) -> np.ndarray:
        """Network outputs [n][5] in scaled units (tensor-core kernel)."""
        X = _f32(X)
        Y = np.empty((X.shape[0], NOUT), dtype=np.float32)
        N.check(self._lib.titan_mlp_forward(N.ptr(self.params, N.F32), N.ptr(self.norm, N.F32), N.ptr(X, N.F32),
                                            X.shape[0], N.ptr(Y, N.F32)))
        return Y

    def predict(self, state: np.ndarray, cc: np.ndarray) -> np.ndarray:
        """Sources [5][n] (n_H, S_m, S_E) for a state and its cell centres."""
        Y = self.forward(features(state, cc, self.n_inf, self.lam)).astype(np.float64)
        return sources(state, cc, Y * self.norm[2 * NIN:], self.n_inf, self.lam)

    def install(self, step) -> None:
        """Every later step of `step` (a PlasmaStep) takes its sources from this network."""
        N.check(self._lib.titan_set_closure(step.ctx, N.ptr(self.params, N.F32), N.ptr(self.norm, N.F32),
                                            self.n_inf, self.lam))

    @staticmethod
    def uninstall(step) -> None:
        N.check(N.lib().titan_set_closure(step.ctx, None, None, 0.0, 0.0))


def run_coupled(step, net: Closure, steps: int, mc_every: int = 100, **mc) -> dict:
    """The coupled loop of the large configuration: MLP sources every step,
    and every `mc_every` steps a Monte-Carlo pass through the current plasma
    whose sources the cells outside the training envelope use until the next
    pass. mc: the keyword arguments of PlasmaStep.mc_sources."""
    net.install(step)
    net.set_fallback(step, None)  # the envelope; the table comes from each pass
    done, passes, outside = 0, 0, []
    while done < steps:
        step.mc_pass(seed=passes + 1, **mc)
        net.fallback_from_mc(step)
        passes += 1
        k = min(mc_every, steps - done)
        step.go(k)
        done += k
        outside.append(Closure.outside(step))
    return {"steps": done, "mc_passes": passes, "outside_last_step": outside}
