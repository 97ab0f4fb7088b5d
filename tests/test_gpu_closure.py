"""The learned charge-exchange closure on the GPU: the BF16 tensor-core
training gradient against the CPU network oracle, the tcgen05 inference kernel
against the oracle's forward pass, training that lowers the loss, the closure
inside the plasma step, and a trained closure judged against Monte-Carlo noise
(what the network gains over holding the last Monte-Carlo sources fixed)."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mlp_oracle as mo  # noqa: E402


def _rand_problem(titan, n, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, 8)).astype(np.float32) * 2.0 + 1.0
    norm = np.concatenate([np.full(8, 1.0), np.full(8, 0.5), np.ones(5)]).astype(np.float32)
    c = titan.closure.Closure(0.18, 4.0, norm=norm, seed=seed)
    c.params += (0.02 * rng.standard_normal(c.params.size) * (c.params != 0)).astype(np.float32)
    for w, b, i, j in mo.offsets():     # non-zero biases (padding stays zero)
        live = j if j == 128 else 5
        c.params[b:b + live] = 0.05 * rng.standard_normal(live)
    T = rng.standard_normal((n, 5)).astype(np.float32)
    return c, X, T


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("n", [1, 200, 1001, 8192])
def test_training_gradient_matches_the_cpu_oracle(titan, n):
    c, X, T = _rand_problem(titan, n, seed=n)
    w = np.array([1.0, 0.5, 2.0, 1.0, 0.25], np.float32)
    rw = None if n % 2 == 0 else np.random.default_rng(n).uniform(0.1, 3.0, n).astype(np.float32)
    loss, g, Y = c.grad(X, T, w, row_weights=rw)
    lo, go = mo.loss_grad(c.params, c.norm, X, T, w, emulate_bf16=True, row_w=rw)
    Yo, _ = mo.forward(c.params, c.norm, X, emulate_bf16=True)
    assert _rel(Y, Yo) < 2e-3
    assert abs(loss - lo) <= 2e-3 * lo
    for li, (wo, bo, i, j) in enumerate(mo.offsets()):
        assert _rel(g[wo:bo], go[wo:bo]) < 1e-2, ("W", li, _rel(g[wo:bo], go[wo:bo]))
        assert _rel(g[bo:bo + j], go[bo:bo + j]) < 1e-2, ("b", li)


@pytest.mark.parametrize("n", [1, 127, 128, 129, 5000, 300_000])
def test_tensor_core_inference_matches_the_oracle(titan, n):
    """tcgen05 forward (activations as BF16 hi/lo pairs, SiLU in FP32 through
    tanh.approx.f32) against the oracle's inference model (BF16 weights,
    full-precision activations) to 1e-3, and against its BF16-rounded training
    forward to the BF16 rounding of the activations; two launches on the same
    input agree bit for bit (the kernel has no order-dependent arithmetic)."""
    c, X, _ = _rand_problem(titan, n, seed=7)
    Y = c.forward(X)
    m = min(n, 20000)
    Yi, _ = mo.forward(c.params, c.norm, X[:m], inference=True)
    Yo, _ = mo.forward(c.params, c.norm, X[:m], emulate_bf16=True)
    assert np.isfinite(Y).all()
    assert _rel(Y[:m], Yi) < 1e-3, _rel(Y[:m], Yi)
    assert _rel(Y[:m], Yo) < 3e-2, _rel(Y[:m], Yo)
    assert np.array_equal(c.forward(X), Y)
    # the GEMM path (training forward) agrees with the same accuracy
    _, _, Yg = c.grad(X[:m], np.zeros((m, 5), np.float32))
    assert _rel(Y[:m], Yg) < 3e-2


def test_training_lowers_the_loss(titan):
    rng = np.random.default_rng(2)
    n = 32768
    X = rng.standard_normal((n, 8)).astype(np.float32)
    T = np.stack([np.sin(X[:, 0]) + X[:, 1] * X[:, 2], np.tanh(X[:, 3]), X[:, 4] ** 2 - 1.0,
                  np.cos(X[:, 5] + X[:, 6]), X[:, 7] * X[:, 0]], axis=1).astype(np.float32)
    c = titan.closure.Closure(0.18, 4.0, seed=1)
    losses = c.fit(X, T, epochs=12, batch=1024, lr=2e-3, lr_decay=0.85)
    assert losses[-1] < 0.1 * losses[0], losses
    assert np.isfinite(c.params).all()
    # padding stays zero
    w1 = c.params[:16 * 128].reshape(16, 128)
    assert not w1[8:].any()


def _shell_run(titan, steps, nq=10, nlayer=14):
    m, p, st, _ = titan.problems.heliosphere_shell(nq=nq, nlayer=nlayer, move=False)
    g = titan.PlasmaStep(m, p)
    g.upload_state(st)
    return m, p, g


def test_closure_inside_the_step_equals_its_sources(titan):
    """A step with the network installed changes the state as a step given
    the same network's sources through titan_set_sources does. The kernel
    forms the features in FP32 and numpy in FP64; a feature that lands on the
    other side of a BF16 rounding boundary moves that cell's output by a BF16
    step, so the source-driven changes are compared to 2e-2 (L2, relative)."""
    m, p, g = _shell_run(titan, 0)
    g.go(5)
    st0 = g.download_state()
    dt0, t0 = g.dt, g.t
    cc = g.geometry()["cell_center"].T
    c, _, _ = _rand_problem(titan, 10, seed=3)
    c.norm[:16] = np.concatenate([np.zeros(8), np.ones(8)])
    c.norm[16:] = 1e-3
    S = c.predict(st0, cc)

    def one_step(setup):
        g.upload_state(st0)
        g.dt, g.t = dt0, t0
        setup()
        g.go(1)
        return g.download_state()

    plain = one_step(lambda: None)
    a = one_step(lambda: c.install(g))
    c.uninstall(g)
    b = one_step(lambda: g.set_sources(np.ascontiguousarray(S[1:])))
    g.close()
    for k in (1, 2, 3, 4):
        da, db = a[k] - plain[k], b[k] - plain[k]
        assert np.linalg.norm(db) > 0.0
        rel = np.linalg.norm(da - db) / np.linalg.norm(db)
        assert rel < 2e-2, (k, rel)


def test_trained_closure_beats_fixed_sources_against_a_denoised_target(titan):
    """Train on Monte-Carlo sources of three plasma snapshots, judge on a
    fourth against a denoised target: the mean of 32 Monte-Carlo seeds of
    that snapshot. Errors are volume-weighted L1 over cells (the sources enter
    the conserved variables as S V); rows are weighted by cell volume in
    training too, since the Monte-Carlo samples a cell in proportion to the
    neutral path length inside it. Asserted:
    * the closure beats the method without it — the previous snapshot's
      Monte-Carlo sources held fixed, which is what the plasma loop uses
      between Monte-Carlo passes;
    * the closure is closer to the denoised target than one fresh
      Monte-Carlo pass (a single seed at the training particle count)."""
    m, p, g = _shell_run(titan, 0, nq=10, nlayer=14)
    kw = dict(n_H=0.18, u_H=(-2.6, 0.0, 0.0), cp_H=1.424, n_particles=1_000_000)
    geo = g.geometry()
    cc, vol = geo["cell_center"].T, geo["cell_volume"]
    snaps = []
    for s in range(4):
        g.go(60)
        st = g.download_state()
        nseed = 32 if s == 3 else 2
        seeds = [g.mc_sources(seed=100 * s + k, **kw)[0] for k in range(nseed)]
        snaps.append((st, np.mean(seeds, axis=0), seeds))
    g.close()
    # the generator has charge exchange only, which conserves the neutrals:
    # the cold-model proxy is flat (lambda = 0)
    n_inf, lam = 0.18, 0.0
    X = np.concatenate([titan.closure.features(st, cc, n_inf, lam) for st, _, _ in snaps[:3]])
    # train on single seeds (noisy labels, as the generator gives them)
    T = np.concatenate([titan.closure.targets(st, cc, sd[0], n_inf, lam) for st, _, sd in snaps[:3]])
    c = titan.closure.Closure(n_inf, lam, seed=0)
    losses = c.fit(X, T, epochs=60, batch=2048, lr=2e-3, lr_decay=0.95, row_weights=np.tile(vol, 3))
    assert losses[-1] < losses[0]
    st, target, seeds = snaps[3]
    pred = c.predict(st, cc)

    def l1(a, b):
        return float((np.abs(a[1:5] - b[1:5]) * vol).sum() / (np.abs(b[1:5]) * vol).sum())

    err = l1(pred, target)
    # one seed's distance to the 32-seed mean, corrected to its distance to the truth
    one_pass = np.mean([l1(sd, target) for sd in seeds[:8]]) * np.sqrt(32.0 / 31.0)
    stale = l1(snaps[2][2][0], target)
    print(f"closure {err:.3e}  one fresh Monte-Carlo pass {one_pass:.3e}  "
          f"previous snapshot's sources held fixed {stale:.3e}")
    assert err < stale
    assert err < one_pass


def test_cells_outside_the_training_envelope_take_the_fallback_sources(titan):
    """With an envelope that cuts the shell between two layers, the outer
    cells take the fallback table (a Monte-Carlo pass's sources) exactly, the
    inner ones the network, and the library counts the outer ones."""
    m, p, g = _shell_run(titan, 0)
    g.go(3)
    st0 = g.download_state()
    dt0, t0 = g.dt, g.t
    cc = g.geometry()["cell_center"].T
    r = np.linalg.norm(cc, axis=0)
    logs = np.sort(np.unique(np.round(np.log(r), 2)))   # one value per radial layer
    k = len(logs) // 2
    cut = 0.5 * (logs[k] + logs[k + 1])
    out_mask = np.log(r) > cut
    assert 0 < out_mask.sum() < len(r)
    c, _, _ = _rand_problem(titan, 10, seed=4)
    c.norm[:16] = np.concatenate([np.zeros(8), np.ones(8)])
    c.norm[16:] = 1e-3
    lo = np.full(8, -3e38, np.float32)
    hi = np.full(8, 3e38, np.float32)
    hi[4] = cut
    c.envelope = (lo, hi)
    c.margined_envelope = lambda rel=0.0: (lo, hi)   # the cut exactly between two layers
    rng = np.random.default_rng(8)
    F = np.zeros((5, len(r)))
    F[1:5] = 1e-4 * rng.standard_normal((4, len(r))) * st0[0]
    S = c.predict(st0, cc)
    S[1:5, out_mask] = F[1:5, out_mask]

    def one_step(setup):
        g.upload_state(st0)
        g.dt, g.t = dt0, t0
        setup()
        g.go(1)
        return g.download_state()

    plain = one_step(lambda: None)

    def with_closure():
        c.install(g)
        c.set_fallback(g, F)

    a = one_step(with_closure)
    n_out = titan.closure.Closure.outside(g)
    c.uninstall(g)
    b = one_step(lambda: g.set_sources(np.ascontiguousarray(S[1:5])))
    g.close()
    assert n_out == int(out_mask.sum())
    for k in (1, 2, 3, 4):
        da, db = a[k] - plain[k], b[k] - plain[k]
        # outer cells: the fallback sources exactly, so identical updates
        np.testing.assert_allclose(da[out_mask], db[out_mask], rtol=1e-12, atol=1e-300)
        rel = np.linalg.norm(da - db) / np.linalg.norm(db)
        assert rel < 2e-2, (k, rel)


def test_fallback_from_a_device_pass_equals_the_host_table(titan):
    """titan_closure_fallback_from_mc (the pass's sources copied on the device)
    gives the same step as the same pass downloaded and handed back through
    titan_set_closure_fallback; with every cell outside the envelope, the
    step's sources are the pass's exactly (up to the order of the tallies'
    atomic additions)."""
    m, p, g = _shell_run(titan, 0, nq=8, nlayer=10)
    g.go(5)
    st0 = g.download_state()
    dt0, t0 = g.dt, g.t
    kw = dict(n_H=0.18, u_H=(-2.6, 0.0, 0.0), cp_H=1.424, n_particles=300_000, seed=5)
    c, _, _ = _rand_problem(titan, 10, seed=2)
    lo = np.full(8, 1e30, np.float32)     # an empty envelope: every cell outside
    hi = np.full(8, -1e30, np.float32)
    c.envelope = (lo, hi)
    c.margined_envelope = lambda rel=0.0: (lo, hi)

    def one_step(setup):
        g.upload_state(st0)
        g.dt, g.t = dt0, t0
        setup()
        g.go(1)
        return g.download_state()

    host, info = g.mc_sources(**kw)
    assert info["lost"] == 0 and np.abs(host[1:5]).max() > 0

    def via_host():
        c.install(g)
        c.set_fallback(g, host)

    a = one_step(via_host)
    assert titan.closure.Closure.outside(g) == g.ncell
    c.uninstall(g)

    def via_device():
        c.install(g)
        c.set_fallback(g, None)
        g.mc_pass(**kw)
        c.fallback_from_mc(g)

    b = one_step(via_device)
    c.uninstall(g)
    g.close()
    for k in range(8):
        np.testing.assert_allclose(b[k], a[k], rtol=1e-9, atol=1e-13 * np.abs(a[k]).max())


def test_closure_beside_the_face_kernel_gives_the_same_steps(titan):
    """titan_set_closure_overlap: the network on its own stream beside the face
    kernel, or before it; both read only the step's state and the cell update
    waits for both, so the states are identical (graph and single steps)."""
    m, p, st, _ = titan.problems.heliosphere_shell(nq=10, nlayer=8, move=True, flux_precision=32)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    net = titan.closure.Closure.load(os.path.join(root, "titan_c-_b200", "data", "closure_shell.npz"))
    outs = []
    for on in (False, True):
        for chunks in ([4], [1, 1, 1, 1]):
            g = titan.PlasmaStep(m, p)
            g.upload_state(st)
            net.install(g)
            g.set_closure_overlap(on)
            for k in chunks:
                g.go(k)
            outs.append(g.download_state())
            g.close()
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
