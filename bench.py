"""Benchmark of the B200 plasma step: MHD cell-updates/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--mode mixed-mlp|fp64|fp32] [--nq 96] [--nlayer 40]

Workload (N=1): the heliosphere-like shell — cubed sphere 6x96x96 x 40
geometric layers = 2,211,840 hexahedra, r in [1, 100], supersonic Parker-spiral
wind inside, interstellar inflow outside, seeded lognormal perturbation,
HLLD where B^2/(8 pi p) > 0.01 else HLLC, prescribed radial node motion (ALE).
One step = one pass of the plasma loop over every face and cell.

Modes: coupled — the large configuration's loop: the mixed step with MLP
sources every step and a Monte-Carlo pass (1e7 particles) every 100 steps
whose sources the cells outside the closure's training envelope use.
mixed-mlp (default) — FP32 Riemann flux with FP64 accumulation, dt and
pressure recovery, and charge-exchange sources from the MLP closure on the
tensor cores every step; the same run also times the plain all-FP64 step on
the same mesh and measures the mixed step's error against it after 100 and
1000 steps (the FP64 GPU step equals the FP64 oracle per step). fp64 / fp32:
the plain step alone at that flux precision.

value: cell-updates/s with the state resident in HBM (device events around K
steps on the library's stream). e2e: the same metric through the C ABI with
host buffers — every step uploads the full cell state from pinned host memory,
steps once and downloads the new state. Inputs (state 141 MB + face data) are
larger than the 126 MB L2, so no flush is needed between steps.
--impl reference: the CPU oracle (restatement of Setka::Go's plasma loop,
OpenMP over all host cores) on the same workload, a bounded number of steps.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "MHD cell-updates/s on 1 B200, mixed/NN-source vs plain FP64 at stated error"
UNIT = "cell-updates/s"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def peak_tflops():
    """Dense BF16 tensor peak measured with cuBLAS, TFLOP/s: the sustained
    figure, since the closure kernel runs inside a long step loop."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops_sustained"]), "measured (sustained)"
    except Exception:
        return 1400.0, "fallback (sustained)"


# DRAM bytes (read + write) per launch from one ncu capture of the kernel on the
# 6x64x64x40 shell, scaled by faces (x2.25) to the 6x96x96x40 workload:
# profiles/face_flux_shell.md has the command and the figures.
TRAFFIC = {("face_flux_fp64", 2211840): 1264.7e6, ("face_flux_fp32", 2211840): 987.7e6}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows]
        smax = float(rows[0][2])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


def build_problem(args):
    pkg = importlib.import_module("titan_c-_b200")
    m, p, st, _ = pkg.problems.heliosphere_shell(nq=args.nq, nlayer=args.nlayer, move=True,
                                                 flux_precision=64 if args.mode == "fp64" else 32)
    return pkg, m, p, st


NET_PATH = os.path.join(ROOT, "titan_c-_b200", "data", "closure_shell.npz")


def load_closure(pkg, m, st):
    """The closure network of the shell problem: the trained one when it is
    present, else the architecture with seeded random weights (the step's cost
    does not depend on the weights) and output scales of a plausible size."""
    cl = pkg.closure
    if os.path.exists(NET_PATH):
        return cl.Closure.load(NET_PATH), "trained"
    cc = m["node_xyz"][m["cell_nodes"]].mean(axis=1).T
    X = cl.features(st, cc, 0.18, 0.0)
    norm = cl.make_norm(X, np.ones((1, 5)))
    norm[16:] = 1e-3
    return cl.Closure(0.18, 0.0, norm=norm, seed=0), "random-init"


def rel_errors(a, b):
    """Relative L1 and Linf of rho, p and |B| of state a against state b."""
    out = {}
    fields = {"rho": (a[0], b[0]), "p": (a[4], b[4]),
              "B": (np.linalg.norm(a[5:8], axis=0), np.linalg.norm(b[5:8], axis=0))}
    for k, (x, y) in fields.items():
        d = np.abs(x - y)
        out[k] = {"l1": float(d.sum() / np.abs(y).sum()), "linf": float(d.max() / np.abs(y).max())}
    return out


def error_study(pkg, m, p, st, tuning, closure, checkpoints=(100, 1000)):
    """Error of the mixed step (FP32 Riemann arithmetic) against the all-FP64 step.

    * over_run: both from the same initial state, states compared at each
      checkpoint, with the closure installed in both or in neither;
    * fp64_sensitivity: the FP64 step against itself from an initial state
      perturbed by 1e-7 relative (seeded) — how far an FP32-sized difference
      carries in this flow by the same checkpoints (shocks and floors make the
      run-to-run spread itself of order 1e-4 .. 1e-3 after ~150 steps);
    * one_step: one step of each from identical states taken along the FP64
      run, |mixed - FP64| relative to |FP64 step change| (the precision the
      flux arithmetic itself delivers per step)."""
    res = {"over_run": {}}

    def make(flux, net=None):
        prm = dict(p)
        prm["flux_precision"] = flux
        g = pkg.PlasmaStep(m, prm)
        g.set_tuning(tuning["face_variant"], tuning["cell_variant"])
        if net is not None:
            net.install(g)
        return g

    def trajectory(flux, s0, net=None):
        g = make(flux, net)
        g.upload_state(s0)
        done, out = 0, {}
        for c in checkpoints:
            g.go(c - done)
            done = c
            out[c] = (g.download_state(), g.dt, g.t)
        g.close()
        return out

    ref = trajectory(64, st)
    for tag, net in (("no_sources", None), ("with_mlp_sources", closure)):
        r64 = ref if net is None else trajectory(64, st, net)
        r32 = trajectory(32, st, net)
        res["over_run"][tag] = {str(c): rel_errors(r32[c][0], r64[c][0]) for c in checkpoints}
    rng = np.random.default_rng(1)
    pert = trajectory(64, st * (1.0 + 1e-7 * rng.standard_normal(st.shape)))
    res["fp64_sensitivity"] = {"perturbation": 1e-7,
                               **{str(c): rel_errors(pert[c][0], ref[c][0]) for c in checkpoints}}
    g64, g32 = make(64), make(32)
    res["one_step"] = {}
    for c in (0,) + tuple(checkpoints):
        s0, dt, t = (st, 1e-5, 0.0) if c == 0 else ref[c]
        outs = []
        for g in (g64, g32):
            g.upload_state(s0)
            g.dt, g.t = dt, t
            g.go(1)
            outs.append(g.download_state())
        d64 = outs[0] - s0
        e = {}
        for k, i in (("rho", 0), ("p", 4)):
            e[k] = float(np.abs(outs[1][i] - outs[0][i]).sum() / max(np.abs(d64[i]).sum(), 1e-300))
        db = np.linalg.norm(outs[1][5:8] - outs[0][5:8], axis=0).sum()
        e["B"] = float(db / max(np.linalg.norm(d64[5:8], axis=0).sum(), 1e-300))
        res["one_step"][f"from_step_{c}"] = e
    g64.close()
    g32.close()
    return res


def face_flux_bytes(m, move: bool, fp32: bool) -> float:
    """Algorithmic DRAM bytes of one face-flux launch: every input read once,
    every output written once — face data, the two cells' states, the node
    coordinates of both layers when the mesh moves, and the 9 FP64 flux values
    of each face (the record's 8-byte pad is not counted)."""
    C = m["cell_nodes"].shape[0]
    F = m["face_nodes"].shape[0]
    N = m["node_xyz"].shape[0]
    per_face = 8 + 2 + 3 * 8 + 8 + 8      # c0,c1 | type,method | normal | area | half distance
    state = 8 * 8 * C                       # 8 FP64 primitives per cell, read once
    out = (9 * 8) * F                       # 9 fluxes (x area) per face, FP64 records in every mode
    # moving mesh: face node ids + node coordinates of both layers replace the
    # stored normal / area / half distance, and cell centres are read instead
    ale = (16 * F + 2 * 24 * N + 24 * C - 40 * F) if move else 0
    return float(per_face * F + state + out + ale)


def timed_steps(step, steps, barrier, stream, dev):
    """Device time of `steps` steps (ms) with the clocks sampled meanwhile."""
    import torch

    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(dev) as clk:
        ev0.record(stream)
        step.go(steps)
        ev1.record(stream)
        barrier()
    return ev0.elapsed_time(ev1), clk.summary()


def make_step(pkg, m, p, st, flux, tuning_arg, closure=None):
    prm = dict(p)
    prm["flux_precision"] = flux
    step = pkg.PlasmaStep(m, prm)
    step.upload_state(st)
    if closure is not None:
        closure.install(step)
    if tuning_arg == "auto":
        tuning = step.autotune(reps=3)
    else:
        fv, cv = (int(x) for x in tuning_arg.split(","))
        step.set_tuning(fv, cv)
        tuning = step.tuning()
    return step, tuning


def run_ours(args, rank, world):
    import torch

    dev = rank % max(torch.cuda.device_count(), 1)
    torch.cuda.set_device(dev)
    pkg, m, p, st = build_problem(args)
    C = m["cell_nodes"].shape[0]
    F = m["face_nodes"].shape[0]
    flux = 64 if args.mode == "fp64" else 32
    closure, net_kind = (load_closure(pkg, m, st) if args.mode in ("mixed-mlp", "coupled") else (None, None))
    step, tuning = make_step(pkg, m, p, st, flux, args.tuning, closure)
    kernels_per_step = (3 if p["move"] else 2) + (1 if closure is not None else 0)
    flux_name = f"face_flux_fp{flux}"

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # warm-up (also captures the CUDA graph)
    step.go(max(args.warmup, 3))
    stream = torch.cuda.ExternalStream(step.stream())
    coupled = None
    if args.mode == "coupled":
        # the large configuration's loop: MLP sources every step, a Monte-Carlo
        # pass every 100 steps whose sources the out-of-envelope cells use
        mc = dict(n_H=0.18, u_H=(-2.6, 0.0, 0.0), cp_H=float(np.sqrt(2.0 * (0.06 * 1.3 ** 2 / (5.0 / 3.0)) / 0.06)),
                  n_particles=10_000_000)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        barrier()
        with ClockSampler(dev) as clk:
            ev0.record(stream)
            coupled = pkg.closure.run_coupled(step, closure, args.steps, mc_every=100, **mc)
            ev1.record(stream)
            barrier()
        ms, clocks = ev0.elapsed_time(ev1), clk.summary()
    else:
        ms, clocks = timed_steps(step, args.steps, barrier, stream, dev)

    # dominant kernel: per-launch device time with events on the library stream
    step.set_profiling(True)
    step.go(args.steps)
    kt = step.kernel_times()
    step.set_profiling(False)
    k_ms, k_n = kt[flux_name]
    k_avg = k_ms / k_n
    total_k = sum(v[0] for v in kt.values())

    # end to end through the C ABI with pinned host buffers
    host = torch.empty((10, C), dtype=torch.float64, pin_memory=True).numpy()
    host[:] = step.download_state()
    e2e_steps = max(3, min(args.steps, 20))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        step.upload_state(host)
        step.go(1)
        step.download_state(host)
    barrier()
    e2e_wall = time.perf_counter() - t0
    ns = 8 + p["npassive"]
    step.close()

    # the plain all-FP64 step on the same mesh, and the mixed step's error against it
    plain = fp32_only = None
    if args.mode in ("mixed-mlp", "coupled"):
        s64, tun64 = make_step(pkg, m, p, st, 64, args.tuning)
        s64.go(max(args.warmup, 3))
        ms64, clk64 = timed_steps(s64, args.steps, barrier, torch.cuda.ExternalStream(s64.stream()), dev)
        s64.close()
        plain = {"value": world * C * args.steps / (ms64 / 1e3), "ms_per_step": ms64 / args.steps,
                 "tuning": tun64, "clocks": clk64}
        # and the FP32-flux step without the closure (the mixed step's other half)
        s32, tun32 = make_step(pkg, m, p, st, 32, args.tuning)
        s32.go(max(args.warmup, 3))
        ms32, clk32 = timed_steps(s32, args.steps, barrier, torch.cuda.ExternalStream(s32.stream()), dev)
        s32.close()
        fp32_only = {"ms_per_step": ms32 / args.steps, "tuning": tun32, "clocks": clk32}

    t = torch.tensor([ms, e2e_wall] + ([plain["ms_per_step"], fp32_only["ms_per_step"]] if plain else []),
                     dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms, e2e_wall = float(t[0]), float(t[1])
    if plain:
        plain["ms_per_step"] = float(t[2])
        plain["value"] = world * C / (plain["ms_per_step"] / 1e3)
        fp32_only["ms_per_step"] = float(t[3])
        fp32_only["value"] = world * C / (fp32_only["ms_per_step"] / 1e3)
    if rank != 0:
        return None
    value = world * C * args.steps / (ms / 1e3)
    hbm, src = peaks()
    bytes_launch = face_flux_bytes(m, bool(p["move"]), flux == 32)
    achieved = bytes_launch / (k_avg / 1e3) / 1e9
    dtype = {"fp64": "f64", "fp32": "f32-flux/f64-update", "mixed-mlp": "f32-flux/f64-update, bf16 MLP",
             "coupled": "f32-flux/f64-update, bf16 MLP, f64 Monte-Carlo"}[args.mode]
    what = {"fp64": "FP64 flux", "fp32": "FP32 flux, FP64 accumulation",
            "mixed-mlp": "FP32 flux, FP64 accumulation, MLP charge-exchange sources every step",
            "coupled": "FP32 flux, FP64 accumulation, MLP sources every step, Monte-Carlo (1e7 particles) "
                       "fallback for out-of-envelope cells every 100 steps"}[args.mode]
    traffic = TRAFFIC.get((flux_name, C))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": dtype,
        "data": "synthetic (seeded heliosphere-like shell; no external data)",
        "config": {"workload": f"heliosphere shell 6x{args.nq}x{args.nq}x{args.nlayer} = {C} cells, {F} faces, "
                               f"ALE, HLLD/HLLC, {what}", "cells": C, "faces": F, "mode": args.mode,
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU", "tuning": tuning,
                   "l2": f"inputs larger than L2 (state {8 * ns * C / 1e6:.0f} MB + face records "
                         f"{80 * F / 1e6:.0f} MB per step), no flush"},
        "face_fluxes_per_s": world * F * args.steps / (ms / 1e3),
        "e2e": {"value": world * C * e2e_steps / e2e_wall, "unit": UNIT,
                "h2d_bytes_per_step": 8 * ns * C, "d2h_bytes_per_step": 8 * ns * C},
        "gpu_launches": args.steps * kernels_per_step,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": traffic, "traffic_source": "ncu capture at 6x64x64x40 scaled by faces" if traffic else None,
                     "kernel": flux_name, "peak_source": src,
                     "algorithmic_bytes_per_launch": bytes_launch, "avg_launch_ms": k_avg,
                     "kernel_share": k_ms / total_k},
        "kernel_ms_per_step": {k: v[0] / v[1] for k, v in kt.items()},
        "clocks": clocks,
    }
    if closure is not None:
        mlp_ms = kt["closure_mlp"][0] / kt["closure_mlp"][1]
        flops = 2.0 * C * (16 * 128 + 3 * 128 * 128 + 128 * 16)
        tf_peak, tf_src = peak_tflops()
        if coupled is not None:
            line["coupled"] = {"mc_passes": coupled["mc_passes"], "mc_every": 100,
                               "cells_outside_envelope": coupled["outside_last_step"]}
            line["gpu_launches"] = args.steps * kernels_per_step + 2 * coupled["mc_passes"]
        line["closure"] = {"network": net_kind, "kernel": "closure_mlp (tcgen05, TMEM accumulators)",
                           "avg_launch_ms": mlp_ms, "flops_per_launch": flops,
                           "tflops": flops / (mlp_ms / 1e3) / 1e12, "tensor_peak_tflops": tf_peak,
                           "peak_source": tf_src, "tensor_frac": flops / (mlp_ms / 1e3) / 1e12 / tf_peak}
    if plain:
        line["plain_fp64"] = plain
        line["fp32_flux_no_closure"] = fp32_only
        line["speedup_vs_plain_fp64"] = plain["ms_per_step"] / (ms / args.steps)
        if world == 1 and args.error_study:
            line["error_vs_fp64"] = error_study(pkg, m, p, st, tuning, closure)
    if args.cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(args, m, p, st)
    return line


def cpu_baseline(args, m, p, st, steps=None):
    """The oracle (OpenMP restatement of Setka::Go's plasma loop) on the same
    mesh, a bounded number of steps."""
    import oracle_lib as ol

    run = ol.OracleRun(m, p)
    s = np.ascontiguousarray(st.copy())
    steps = steps or args.cpu_steps
    run.go(s, 1)  # first touch / geometry warm-up
    t0 = time.perf_counter()
    run.go(s, steps)
    dt = time.perf_counter() - t0
    C = m["cell_nodes"].shape[0]
    return {"value": C * steps / dt, "unit": UNIT, "cores": int(ol.oracle().oracle_num_threads()),
            "kind": "port", "sample": f"{steps} steps of the full {C}-cell workload "
                                      f"({dt:.1f} s), oracle/titan_oracle.cpp with OpenMP"}


def run_sharded(args, rank, world):
    """One shell split over the ranks (titan.shard: Morton ranges, one-cell halo
    exchanged over NCCL each step, dt as the minimum over the ranks): strong
    scaling of the FP64 or FP32-flux step. Opt-in (--shard); without it,
    --gpus N runs N replicas."""
    import torch

    if args.mode == "coupled":
        raise SystemExit("--shard runs the fp64, fp32 or mixed-mlp step (the Monte-Carlo is not sharded)")
    dev = rank % max(torch.cuda.device_count(), 1)
    torch.cuda.set_device(dev)
    pkg, m, p, st = build_problem(args)
    C = m["cell_nodes"].shape[0]
    flux = 64 if args.mode == "fp64" else 32
    ss = pkg.shard.ShardedStep(pkg, m, dict(p, flux_precision=flux), rank, world, torch.device("cuda", dev))
    ss.upload_state(st)
    plasma = ss.step.step
    if args.mode == "mixed-mlp":
        # the closure runs per rank on its sub-mesh's cells
        closure, _ = load_closure(pkg, m, st)
        closure.install(plasma)
    tuning = plasma.autotune(reps=3) if args.tuning == "auto" else None
    kernels = (3 if p["move"] else 2) + (1 if args.mode == "mixed-mlp" else 0)
    kernels += (1 if ss.n_send else 0) + (1 if ss.n_recv else 0)  # halo pack / unpack

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    ss.go(max(args.warmup, 3))
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(dev) as clk:
        ev0.record()
        ss.go(args.steps)
        ev1.record()
        barrier()
    # end to end: every step each rank's cells in from pinned host memory, the owned cells back
    ns = 8 + p["npassive"]
    n_loc = len(ss.shard["cells"])
    host = torch.empty((10, n_loc), dtype=torch.float64, pin_memory=True).numpy()
    host[:] = st[:, ss.shard["cells"]]
    e2e_steps = max(3, min(args.steps, 20))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        plasma.upload_state(host)
        ss.go(1)
        plasma.download_state(host)
    barrier()
    e2e_wall = time.perf_counter() - t0
    t = torch.tensor([ev0.elapsed_time(ev1), e2e_wall], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms, e2e_wall = float(t[0]), float(t[1])
    clocks = clk.summary()
    ss.close()
    if rank != 0:
        return None
    value = C * args.steps / (ms / 1e3)
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": {"fp64": "f64", "fp32": "f32-flux/f64-update", "mixed-mlp": "f32-flux/f64-update, bf16 MLP"}[args.mode],
        "data": "synthetic (seeded heliosphere-like shell; no external data)",
        "config": {"workload": f"heliosphere shell 6x{args.nq}x{args.nq}x{args.nlayer} = {C} cells split over "
                               f"{world} GPUs (Morton ranges, one-cell halo over NCCL)",
                   "cells": C, "mode": args.mode, "parallelism": f"sharded x{world}", "tuning": tuning},
        "e2e": {"value": C * e2e_steps / e2e_wall, "unit": UNIT,
                "h2d_bytes_per_step": 8 * ns * n_loc, "d2h_bytes_per_step": 8 * ns * n_loc,
                "note": "rank 0's bytes; every rank moves its own cells"},
        "gpu_launches": kernels * args.steps, "clocks": clocks,
    }


def run_reference(args, rank, world):
    if rank != 0:
        return None
    pkg, m, p, st = build_problem(args)
    C = m["cell_nodes"].shape[0]
    import oracle_lib as ol

    run = ol.OracleRun(m, p)
    s = np.ascontiguousarray(st.copy())
    run.go(s, max(args.warmup, 1))
    t0 = time.perf_counter()
    run.go(s, args.steps)
    dt = time.perf_counter() - t0
    v = C * args.steps / dt
    cores = int(ol.oracle().oracle_num_threads())
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded heliosphere-like shell)",
            "config": {"workload": f"heliosphere shell 6x{args.nq}x{args.nq}x{args.nlayer} = {C} cells, ALE, "
                                   "HLLD/HLLC, FP64", "cells": C},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{args.steps} steps of the full workload after {args.warmup} warm-up"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nq", type=int, default=96)
    ap.add_argument("--nlayer", type=int, default=40)
    ap.add_argument("--mode", default="mixed-mlp", choices=["mixed-mlp", "fp64", "fp32", "coupled"])
    ap.add_argument("--no-error-study", dest="error_study", action="store_false")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--tuning", default="auto", help="auto, or 'face_variant,cell_variant'")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--shard", action="store_true",
                    help="split one mesh over the GPUs (strong scaling) instead of N replicas")
    args = ap.parse_args()
    if args.impl == "reference":
        # a bounded sample of the workload: a full step is about 0.35 s on 16 host threads
        args.steps = min(args.steps, 3)
        args.warmup = min(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and args.impl == "ours":
        import torch
        import datetime

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", rank)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    elif args.shard:
        line = run_sharded(args, rank, world)
    else:
        line = run_ours(args, rank, world)
    if world > 1 and args.impl == "ours":
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
