"""CPU oracle of the charge-exchange closure network (test infrastructure only).

Forward pass, weighted-MSE loss and its gradient for the MLP
8 -> 128 -> 128 -> 128 -> 128 -> 5 (SiLU) in numpy float64, with BF16 rounding
applied at the points where the GPU training path stores BF16 values (the
standardised inputs, the weight copies, the activations and the
back-propagated pre-activation gradients), so the GPU gradient can be checked
to the accuracy of its FP32 accumulation rather than to BF16 precision.

The closure has no counterpart in the reference (it stands in for re-running
the Monte-Carlo neutral solver of TITAN/source/Setka_MK.cpp), so this module is
pinned by construction: a finite-difference check of its own gradient
(tests/test_closure_cpu.py) and the GPU gradient against it.

Parameter vector layout (FP32 masters, 53,776 floats):
[W1 16x128 | b1 128 | W2 128x128 | b2 | W3 | b3 | W4 | b4 | W5 128x16 | b5 16],
each W stored [in][out]; input rows 8..15 of W1 and output columns 5..15 of
W5 / b5 are padding.
"""
from __future__ import annotations

import numpy as np

NIN, NIN_PAD, NHID, NOUT, NOUT_PAD = 8, 16, 128, 5, 16
LAYERS = [(NIN_PAD, NHID), (NHID, NHID), (NHID, NHID), (NHID, NHID), (NHID, NOUT_PAD)]


def offsets():
    """[(w_offset, b_offset, in, out)] per layer."""
    out, o = [], 0
    for i, j in LAYERS:
        out.append((o, o + i * j, i, j))
        o += i * j + j
    return out


NPARAM = offsets()[-1][1] + NOUT_PAD


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params: np.ndarray):
    p = np.asarray(params, dtype=np.float64)
    return [(p[w:b].reshape(i, j), p[b:b + j]) for w, b, i, j in offsets()]


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def standardise(X, norm):
    mean, istd = norm[:NIN], norm[NIN:2 * NIN]
    x0 = np.zeros((X.shape[0], NIN_PAD))
    x0[:, :NIN] = (np.asarray(X, np.float32) - mean.astype(np.float32)) * istd.astype(np.float32)
    return x0


def forward(params, norm, X, emulate_bf16: bool = True, inference: bool = False):
    """Outputs Y [n][5] (network units) and the cache for backward.

    inference=True models the tcgen05 inference kernel instead of the training
    path: weights and biases rounded to BF16, inputs and activations kept at
    full precision (the kernel carries each as a BF16 hi + lo pair, about 16
    significant bits, and evaluates SiLU in FP32)."""
    r = bf16 if emulate_bf16 and not inference else (lambda a: np.asarray(a, np.float64))
    a = r(standardise(X, norm))
    cache = {"A": [a], "Z": [], "W": []}
    layers = unpack(params)
    for li, (W, b) in enumerate(layers):
        Wr = bf16(W) if inference else r(W)
        if inference:
            b = bf16(b)
        z = a @ Wr + b
        cache["W"].append(Wr)
        cache["Z"].append(z)
        if li < 4:
            a = r(silu(z))
            cache["A"].append(a)
    return cache["Z"][-1][:, :NOUT], cache


def loss_grad(params, norm, X, T, w, emulate_bf16: bool = True, row_w=None):
    """Weighted MSE sum_r rw_r sum_k w_k (Y_rk - T_rk)^2 / n and its gradient [NPARAM]."""
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float64))
    n = X.shape[0]
    Y, c = forward(params, norm, X, emulate_bf16)
    d = Y - T
    rw = np.ones((n, 1)) if row_w is None else np.asarray(row_w, np.float64).reshape(n, 1)
    loss = float((rw * np.asarray(w) * d * d).sum() / n)
    dz = np.zeros((n, NOUT_PAD))
    dz[:, :NOUT] = 2.0 * rw * np.asarray(w) * d / n
    dz = r(dz)
    g = np.zeros(NPARAM)
    offs = offsets()
    for li in range(4, -1, -1):
        wo, bo, i, j = offs[li]
        g[wo:bo] = (c["A"][li].T @ dz).ravel()
        g[bo:bo + j] = dz.sum(axis=0)
        if li > 0:
            da = dz @ c["W"][li].T
            dz = r(da * dsilu(c["Z"][li - 1]))
    return loss, g
