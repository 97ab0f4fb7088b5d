"""Trains the charge-exchange closure of the heliosphere shell on Monte-Carlo
sources and judges it against the Monte-Carlo noise.

    python titan_c-_b200/train_closure.py [--nq 96] [--nlayer 40] [--steps 1000]
        [--snapshots 4] [--particles 1e7] [--seeds 32] [--epochs 12]
        [--out titan_c-_b200/data/closure_shell.npz] [--report FILE.json]

1. The plain FP64 step runs the shell problem (moving mesh) for `steps` steps;
   at `snapshots` evenly spaced steps the plasma state and cell centres are
   kept and the Monte-Carlo neutral solver (PlasmaStep.mc_sources) runs
   through them: one seed per training snapshot, `seeds` independent seeds on
   the last one.
2. The split is by snapshot: all but the last train, the last is held out.
3. The network trains on the GPU (BF16 tensor-core forward/backward, Adam).
4. On the held-out snapshot, against the mean of its seeds (a denoised
   target: 32 seeds by default): the closure's error, one fresh Monte-Carlo
   pass's error (a single seed, corrected for its share of the mean), and the
   error of the method without the closure — the previous snapshot's
   Monte-Carlo sources held fixed (all volume-weighted L1, relative); and the
   time of one Monte-Carlo pass against one closure launch.
Training rows are weighted by cell volume: the Monte-Carlo samples a cell in
proportion to the neutral path length inside it.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _pkg():
    root = os.path.dirname(HERE)
    if root not in sys.path:
        sys.path.insert(0, root)
    return importlib.import_module("titan_c-_b200")


def l1(a, b, vol):
    """Volume-weighted L1 difference of the momentum and energy sources,
    relative to b (the sources enter the conserved variables as S V)."""
    return float((np.abs(a[1:5] - b[1:5]) * vol).sum() / (np.abs(b[1:5]) * vol).sum())


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nq", type=int, default=96)
    ap.add_argument("--nlayer", type=int, default=40)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--snapshots", type=int, default=4)
    ap.add_argument("--particles", type=float, default=1e7)
    ap.add_argument("--seeds", type=int, default=32)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--n-inf", type=float, default=0.18)
    ap.add_argument("--lam", type=float, default=0.0)
    ap.add_argument("--out", default=os.path.join(HERE, "data", "closure_shell.npz"))
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)

    pkg = _pkg()
    cl = pkg.closure
    m, p, st, _ = pkg.problems.heliosphere_shell(nq=a.nq, nlayer=a.nlayer, move=True)
    g = pkg.PlasmaStep(m, p)
    g.upload_state(st)
    g.autotune(reps=2)
    # interstellar neutrals: n_H, the interstellar velocity and temperature (cp^2 = 2 p / rho)
    lism_rho, lism_p = 0.06, 0.06 * (2.6 / 2.0) ** 2 / (5.0 / 3.0)
    kw = dict(n_H=a.n_inf, u_H=(-2.6, 0.0, 0.0), cp_H=float(np.sqrt(2.0 * lism_p / lism_rho)),
              n_particles=int(a.particles))
    every = a.steps // a.snapshots
    snaps, mc_ms = [], []
    done = 0
    for k in range(a.snapshots):
        g.go(every * (k + 1) - done)
        done = every * (k + 1)
        state = g.download_state()
        geo = g.geometry()
        cc, vol = geo["cell_center"].T.copy(), geo["cell_volume"].copy()
        nseed = a.seeds if k == a.snapshots - 1 else 1
        runs = []
        for s in range(nseed):
            t0 = time.perf_counter()
            out, info = g.mc_sources(seed=1000 * k + s + 1, **kw)
            mc_ms.append(1e3 * (time.perf_counter() - t0))
            runs.append(out)
        snaps.append({"step": done, "state": state, "cc": cc, "vol": vol, "runs": runs})
        print(f"snapshot step {done}: MC {nseed} seed(s), last {mc_ms[-1]:.0f} ms, lost {info['lost']}",
              flush=True)

    train, test = snaps[:-1], snaps[-1]
    X = np.concatenate([cl.features(s["state"], s["cc"], a.n_inf, a.lam) for s in train])
    T = np.concatenate([cl.targets(s["state"], s["cc"], s["runs"][0], a.n_inf, a.lam) for s in train])
    rw = np.concatenate([s["vol"] for s in train])  # the Monte-Carlo samples a cell in proportion to its volume
    net = cl.Closure(a.n_inf, a.lam, seed=0)
    t0 = time.perf_counter()
    losses = net.fit(X, T, epochs=a.epochs, batch=a.batch, lr=a.lr, lr_decay=0.8, row_weights=rw)
    train_s = time.perf_counter() - t0
    print(f"trained on {X.shape[0]} rows in {train_s:.1f} s; loss {losses[0]:.4f} -> {losses[-1]:.4f}", flush=True)

    mean = np.mean(test["runs"], axis=0)
    t0 = time.perf_counter()
    pred = net.predict(test["state"], test["cc"])
    vol = test["vol"]
    err = l1(pred, mean, vol)
    ns = len(test["runs"])
    noise = float(np.mean([l1(r, mean, vol) for r in test["runs"]]) * np.sqrt(ns / max(ns - 1, 1)))
    stale = l1(train[-1]["runs"][0], mean, vol)
    # closure cost inside the step: one launch of the tensor-core kernel per step
    net.install(g)
    g.set_profiling(True)
    g.go(10)
    kt = g.kernel_times()
    g.close()
    mlp_ms = kt["closure_mlp"][0] / kt["closure_mlp"][1]
    comp = {}
    def l1c(x, y):
        return float((np.abs(x - y) * vol).sum() / (np.abs(y) * vol).sum())

    for i, name in enumerate(["S_mx", "S_my", "S_mz", "S_E"]):
        comp[name] = {"closure": l1c(pred[1 + i], mean[1 + i]),
                      "one_seed_noise": float(np.mean([l1c(r[1 + i], mean[1 + i]) for r in test["runs"]])
                                              * np.sqrt(ns / max(ns - 1, 1)))}
    report = {
        "mesh": f"shell 6x{a.nq}x{a.nq}x{a.nlayer} = {m['cell_nodes'].shape[0]} cells (moving)",
        "snapshots": [s["step"] for s in snaps], "train_snapshots": [s["step"] for s in train],
        "test_snapshot": test["step"], "particles": int(a.particles), "seeds_on_test": ns,
        "rows": int(X.shape[0]), "epochs": a.epochs, "batch": a.batch, "train_s": train_s,
        "loss_first_last": [float(losses[0]), float(losses[-1])],
        "closure_l1": err, "one_seed_noise_l1": noise, "closure_over_noise": err / noise,
        "stale_previous_snapshot_l1": stale, "closure_beats_stale": bool(err < stale),
        "closure_beats_one_pass": bool(err < noise), "per_component": comp,
        "mc_pass_ms": float(np.median(mc_ms)), "closure_kernel_ms": mlp_ms,
        "mc_over_closure_cost": float(np.median(mc_ms)) / mlp_ms,
    }
    print(json.dumps(report, indent=1))
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    np.savez(a.out, params=net.params, norm=net.norm, n_inf=a.n_inf, lam=a.lam,
             envelope_lo=X.min(axis=0), envelope_hi=X.max(axis=0))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)
    return report


if __name__ == "__main__":
    main()
