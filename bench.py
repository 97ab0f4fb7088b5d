"""Benchmark of the B200 plasma step: MHD cell-updates/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--mode mixed-mlp|fp64|fp32|coupled] [--nq 96] [--nlayer 40]
                    [--no-large] [--no-error-study] [--no-cpu-baseline]

Workload (N=1): the heliosphere-like shell — cubed sphere 6x96x96 x 40
geometric layers = 2,211,840 hexahedra, r in [1, 100], supersonic Parker-spiral
wind inside, interstellar inflow outside, seeded lognormal perturbation,
HLLD where B^2/(8 pi p) > 0.01 else HLLC, prescribed radial node motion (ALE).
One step = one pass of the plasma loop over every face and cell.

Modes: mixed-mlp (default) — FP32 Riemann flux with FP64 accumulation, dt and
pressure recovery, and charge-exchange sources from the MLP closure on the
tensor cores every step; the same run times the plain all-FP64 step and the
FP32-flux step without the closure on the same mesh, measures the mixed
step's error against the FP64 step after 100 and 1000 steps, and (unless
--no-large) repeats the mixed and FP64 timings on the 6x192x192x40 shell
(8,847,360 cells). coupled — the large configuration's loop: the mixed step
with MLP sources every step and a Monte-Carlo pass (1e7 particles) every 100
steps whose sources the cells outside the closure's training envelope use.
fp64 / fp32: the plain step alone at that flux precision.

value: cell-updates/s with the state resident in HBM (device events around K
steps on the library's stream). e2e: the same metric through the C ABI with
host buffers — every step uploads the full cell state from pinned host memory,
steps once and downloads the new state. Inputs (state 141 MB + face data) are
larger than the 126 MB L2, so no flush is needed between steps.
roofline: the dominant kernel (largest share of the step's kernel time),
algorithmic bytes (or FLOP) per launch over its event time; step_roofline: the
whole step's algorithmic bytes per cell-update (the scope's definition, face
flux intermediates not counted) over the time per step; kernel_rooflines: the
same for every kernel of the step, with the FP64-pipe ceiling of the FP64
face kernel from its counted instructions.
--impl reference: the CPU oracle (restatement of Setka::Go's plasma loop,
OpenMP over all host cores) on the same workload, up to 100 steps.
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


# DRAM bytes (read + write) per launch, per kernel, from one ncu capture of
# each kernel on the shells themselves (6x96x96x40, the workload of this
# benchmark, and 6x192x192x40, its large shell; ncu --metrics
# dram__bytes_read.sum,dram__bytes_write.sum, one launch each, the launch
# shapes the autotuner picks). Keyed by (kernel, cells, sources in the step);
# other sizes report no traffic.
TRAFFIC = {
    # the mixed step (FP32 Riemann arithmetic, closure sources)
    ("move_nodes", 2211840, True): 107.86e6, ("closure_mlp", 2211840, True): 83.66e6,
    ("face_flux_fp32", 2211840, True): 1039.27e6, ("cell_update", 2211840, True): 1450.35e6,
    ("move_nodes", 8847360, True): 540.41e6, ("closure_mlp", 8847360, True): 427.86e6,
    ("face_flux_fp32", 8847360, True): 4257.45e6, ("cell_update", 8847360, True): 5988.45e6,
    # the plain FP64 step
    ("move_nodes", 2211840, False): 111.87e6, ("face_flux_fp64", 2211840, False): 1045.05e6,
    ("cell_update", 2211840, False): 1163.66e6,
    ("move_nodes", 8847360, False): 543.15e6, ("face_flux_fp64", 8847360, False): 4278.31e6,
    ("cell_update", 8847360, False): 4772.92e6,
}


def traffic(name, C, sources):
    return TRAFFIC.get((name, C, bool(sources)))

# FP64-pipe warp instructions per face of face_flux_fp64 on the moving shell,
# counted by ncu at the benchmark's launch shape (sm__inst_executed_pipe_fp64.sum
# / faces on the 6x64x64x40 shell; 1,173 thread instructions per face: 337 DFMA
# of the IEEE divisions and square roots, 346 DMUL, 268 DADD, the rest compares
# and conversions).
FP64_WARP_INST_PER_FACE = 36.65
FP64_WARP_INST_PER_CLK_PER_SM = 2.0  # 64 FP64 lanes per clock per SM


def step_bytes(m, move: bool, closure: bool):
    """Algorithmic DRAM bytes of one step per cell-update, as the hot-path scope
    defines them: state read + write (2 x 8 x 8), volume, the 6 signed face
    ids of the cell, and per face owner / neighbour ids, normal + area and the
    half distance; a moving mesh adds both layers' node coordinates and the
    new volume; the closure adds its 8 BF16 inputs and 5 FP32 outputs. Face
    flux intermediates are not counted, so fusing them away is rewarded."""
    C = m["cell_nodes"].shape[0]
    F = m["face_nodes"].shape[0]
    N = m["node_xyz"].shape[0]
    b = 2 * 8 * 8 + 8 + 6 * 4 + (F / C) * (2 * 4 + 4 * 8 + 8)
    if move:
        b += 48 * N / C + 8
    if closure:
        b += 8 * 2 + 5 * 4
    return b * C, b


def kernel_work(name: str, m, move: bool, sources: bool):
    """(bound, algorithmic bytes or FLOP per launch) of one step kernel: every
    input it needs read once and every output written once, the face-record
    intermediate between face_flux and cell_update excluded."""
    C = m["cell_nodes"].shape[0]
    F = m["face_nodes"].shape[0]
    N = m["node_xyz"].shape[0]
    if name.startswith("face_flux"):
        if move:   # face node ids, cells, type/surf/method; state and centres; node coordinates of both layers
            return "hbm", float(F * (16 + 8 + 3) + C * (64 + 24) + N * 48)
        return "hbm", float(F * (8 + 3 + 24 + 8 + 8) + C * 64)
    if name == "cell_update":
        b = C * (24 + 64 + 64 + 8 + 2)
        if sources:  # the closure: its 5 FP32 outputs and the centres in, the next step's 8 input words and flag out
            b += C * (20 + 24 + 1 + 32 + 1)
        if move:   # next layer: cell nodes, face->node map, new coordinates; centres and volumes out
            b += C * (32 + 12 + 8 + 24) + N * 24
        return "hbm", float(b)
    if name == "closure_inputs":
        return "hbm", float(C * (40 + 24 + 32 + 1))
    if name == "move_nodes":
        return "hbm", float(N * (24 + 24 + 16))
    if name == "closure_mlp":
        return "tensor", float(C * 2 * (8 * 128 + 3 * 128 * 128 + 128 * 5))
    return "hbm", None


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
    ref_net = None
    for tag, net in (("no_sources", None), ("with_mlp_sources", closure)):
        r64 = ref if net is None else trajectory(64, st, net)
        if net is not None:
            ref_net = r64
        r32 = trajectory(32, st, net)
        res["over_run"][tag] = {str(c): rel_errors(r32[c][0], r64[c][0]) for c in checkpoints}
    rng = np.random.default_rng(1)
    st_p = st * (1.0 + 1e-7 * rng.standard_normal(st.shape))
    pert = trajectory(64, st_p)
    res["fp64_sensitivity"] = {"perturbation": 1e-7,
                               **{str(c): rel_errors(pert[c][0], ref[c][0]) for c in checkpoints}}
    if closure is not None:
        # the same with the closure's sources in both runs
        pn = trajectory(64, st_p, closure)
        res["fp64_sensitivity_with_mlp_sources"] = {
            "perturbation": 1e-7, **{str(c): rel_errors(pn[c][0], ref_net[c][0]) for c in checkpoints}}
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


def measure_mode(pkg, m, p, st, flux, closure, args, barrier, dev, e2e_steps=None):
    """One step configuration on this rank: device time of K steps (events on
    the library's stream, clocks sampled meanwhile), per-kernel launch times,
    and the end-to-end figure through the C ABI with pinned host buffers
    (every step uploads the state, steps once and downloads the new state)."""
    import torch

    step, tuning = make_step(pkg, m, p, st, flux, args.tuning, closure)
    step.go(max(args.warmup, 3))  # warm-up (also captures the CUDA graph)
    stream = torch.cuda.ExternalStream(step.stream())
    ms, clocks = timed_steps(step, args.steps, barrier, stream, dev)
    step.set_profiling(True)
    step.go(args.steps)
    kt = step.kernel_times()
    step.set_profiling(False)
    C = m["cell_nodes"].shape[0]
    host = torch.empty((10, C), dtype=torch.float64, pin_memory=True).numpy()
    host[:] = step.download_state()
    n = e2e_steps or max(3, min(args.steps, 20))
    barrier()
    t0 = time.perf_counter()
    for _ in range(n):
        step.upload_state(host)
        step.go(1)
        step.download_state(host)
    barrier()
    e2e_wall = time.perf_counter() - t0
    step.close()
    return {"ms": ms, "clocks": clocks, "kt": kt, "e2e_wall": e2e_wall, "e2e_steps": n, "tuning": tuning}


def rooflines(kt, m, move, sources, clock_mhz):
    """Per-kernel roofline objects (HBM bytes or tensor FLOP per launch over the
    launch's event time, against the measured peaks) and the dominant kernel
    (largest share of the step's kernel time)."""
    hbm, src = peaks()
    tf, tf_src = peak_tflops()
    C = m["cell_nodes"].shape[0]
    F = m["face_nodes"].shape[0]
    total = sum(v[0] for v in kt.values())
    per = {}
    for name, (tot, n) in kt.items():
        bound, work = kernel_work(name, m, move, sources)
        if work is None or n == 0:
            continue
        avg = tot / n
        if bound == "hbm":
            ach, peak, unit, ps = work / (avg / 1e3) / 1e9, hbm, "GB/s", src
        else:
            ach, peak, unit, ps = work / (avg / 1e3) / 1e12, tf, "TFLOP/s", tf_src
        r = {"bound": bound, "achieved": ach, "peak": peak, "unit": unit, "frac": ach / peak,
             "traffic": traffic(name, C, sources), "kernel": name, "peak_source": ps,
             ("algorithmic_bytes_per_launch" if bound == "hbm" else "algorithmic_flop_per_launch"): work,
             "avg_launch_ms": avg, "kernel_share": tot / total}
        if name == "face_flux_fp64" and clock_mhz:
            ceil = F * FP64_WARP_INST_PER_FACE / (148 * FP64_WARP_INST_PER_CLK_PER_SM * clock_mhz * 1e6) * 1e3
            r["fp64_pipe"] = {"warp_inst_per_face": FP64_WARP_INST_PER_FACE, "ceiling_ms": ceil,
                              "frac": ceil / avg, "clock_mhz": clock_mhz,
                              "note": "time the counted FP64 instructions need at 64 FP64 lanes/clock/SM"}
        per[name] = r
    dominant = max(per, key=lambda k: per[k]["kernel_share"]) if per else None
    return per, dominant


def step_roofline(m, move, closure, ms_per_step, kernels):
    """The whole step against the HBM roofline: the scope's algorithmic bytes per
    cell-update times the cells, over the measured time per step; the DRAM
    traffic per step is the sum of the step kernels' captured traffic."""
    hbm, src = peaks()
    total, per_cell = step_bytes(m, move, closure)
    ach = total / (ms_per_step / 1e3) / 1e9
    C = m["cell_nodes"].shape[0]
    tr = [traffic(k, C, closure) for k in kernels]
    step_traffic = sum(tr) if tr and all(t is not None for t in tr) else None
    return {"bound": "hbm", "bytes_per_cell_update": per_cell, "algorithmic_bytes_per_step": total,
            "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm, "peak_source": src,
            "traffic_per_step": step_traffic,
            "traffic_over_algorithmic": (step_traffic / total) if step_traffic else None}


def run_ours(args, rank, world):
    import torch

    dev = rank % max(torch.cuda.device_count(), 1)
    torch.cuda.set_device(dev)
    pkg, m, p, st = build_problem(args)
    C = m["cell_nodes"].shape[0]
    F = m["face_nodes"].shape[0]
    move = bool(p["move"])
    flux = 64 if args.mode == "fp64" else 32
    use_net = args.mode in ("mixed-mlp", "coupled")
    closure, net_kind = (load_closure(pkg, m, st) if use_net else (None, None))

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    coupled = None
    if args.mode == "coupled":
        # the large configuration's loop: MLP sources every step, a Monte-Carlo
        # pass every 100 steps whose sources the out-of-envelope cells use
        step, tuning = make_step(pkg, m, p, st, flux, args.tuning, closure)
        step.go(max(args.warmup, 3))
        stream = torch.cuda.ExternalStream(step.stream())
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
        step.close()
        head = measure_mode(pkg, m, p, st, flux, closure, args, barrier, dev)
        head["ms"], head["clocks"] = ev0.elapsed_time(ev1), clk.summary()
    else:
        head = measure_mode(pkg, m, p, st, flux, closure, args, barrier, dev)

    # the plain all-FP64 step on the same mesh, and the FP32-flux step without the closure
    plain = fp32_only = None
    if use_net:
        plain = measure_mode(pkg, m, p, st, 64, None, args, barrier, dev)
        fp32_only = measure_mode(pkg, m, p, st, 32, None, args, barrier, dev, e2e_steps=3)

    times = [head["ms"], head["e2e_wall"]]
    if plain:
        times += [plain["ms"], plain["e2e_wall"], fp32_only["ms"]]
    t = torch.tensor(times, dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    t = [float(x) for x in t]
    head["ms"], head["e2e_wall"] = t[0], t[1]
    if plain:
        plain["ms"], plain["e2e_wall"], fp32_only["ms"] = t[2], t[3], t[4]
    if rank != 0:
        return None

    ns = 8 + p["npassive"]
    ms_step = head["ms"] / args.steps
    value = world * C / (ms_step / 1e3)
    clocks = head["clocks"]
    kernels, dominant = rooflines(head["kt"], m, move, use_net, clocks.get("sm_mhz"))
    dtype = {"fp64": "f64", "fp32": "f32-flux/f64-update", "mixed-mlp": "f32-flux/f64-update, bf16 MLP",
             "coupled": "f32-flux/f64-update, bf16 MLP, f64 Monte-Carlo"}[args.mode]
    what = {"fp64": "FP64 flux", "fp32": "FP32 flux, FP64 accumulation",
            "mixed-mlp": "FP32 flux, FP64 accumulation, MLP charge-exchange sources every step",
            "coupled": "FP32 flux, FP64 accumulation, MLP sources every step, Monte-Carlo (1e7 particles) "
                       "fallback for out-of-envelope cells every 100 steps"}[args.mode]
    kernels_per_step = (3 if move else 2) + (1 if use_net else 0)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": dtype,
        "data": "synthetic (seeded heliosphere-like shell; no external data)",
        "config": {"workload": f"heliosphere shell 6x{args.nq}x{args.nq}x{args.nlayer} = {C} cells, {F} faces, "
                               f"ALE, HLLD/HLLC, {what}", "cells": C, "faces": F, "mode": args.mode,
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU", "tuning": head["tuning"],
                   "l2": f"inputs larger than L2 (state {8 * ns * C / 1e6:.0f} MB + face records "
                         f"{80 * F / 1e6:.0f} MB per step), no flush"},
        "face_fluxes_per_s": world * F / (ms_step / 1e3),
        "e2e": {"value": world * C * head["e2e_steps"] / head["e2e_wall"], "unit": UNIT,
                "h2d_bytes_per_step": 8 * ns * C, "d2h_bytes_per_step": 8 * ns * C},
        "gpu_launches": args.steps * kernels_per_step,
        "roofline": kernels.get(dominant),
        "step_roofline": step_roofline(m, move, use_net, ms_step, list(head["kt"])),
        "kernel_rooflines": kernels,
        "kernel_ms_per_step": {k: v[0] / v[1] for k, v in head["kt"].items()},
        "clocks": clocks,
    }
    if use_net:
        cr = kernels.get("closure_mlp", {})
        line["closure"] = {"network": net_kind, "kernel": "closure_mlp (tcgen05, activations in TMEM as BF16 hi/lo)",
                           "avg_launch_ms": cr.get("avg_launch_ms"), "flop_per_launch": cr.get("algorithmic_flop_per_launch"),
                           "tflops": cr.get("achieved"), "tensor_frac": cr.get("frac"),
                           "note": "algorithmic FLOP of the 8-128x4-5 network; the kernel multiplies each "
                                   "activation's BF16 hi and lo halves, twice the tensor work"}
    if coupled is not None:
        line["coupled"] = {"mc_passes": coupled["mc_passes"], "mc_every": 100,
                           "cells_outside_envelope": coupled["outside_last_step"]}
        line["gpu_launches"] = args.steps * kernels_per_step + 2 * coupled["mc_passes"]
    if plain:
        pms = plain["ms"] / args.steps
        pk, pdom = rooflines(plain["kt"], m, move, False, plain["clocks"].get("sm_mhz"))
        line["plain_fp64"] = {
            "value": world * C / (pms / 1e3), "ms_per_step": pms, "tuning": plain["tuning"], "clocks": plain["clocks"],
            "e2e": {"value": world * C * plain["e2e_steps"] / plain["e2e_wall"], "unit": UNIT,
                    "h2d_bytes_per_step": 8 * ns * C, "d2h_bytes_per_step": 8 * ns * C},
            "step_roofline": step_roofline(m, move, False, pms, list(plain["kt"])),
            "roofline": pk.get(pdom), "kernel_rooflines": pk,
            "kernel_ms_per_step": {k: v[0] / v[1] for k, v in plain["kt"].items()}}
        fms = fp32_only["ms"] / args.steps
        line["fp32_flux_no_closure"] = {"value": world * C / (fms / 1e3), "ms_per_step": fms,
                                        "tuning": fp32_only["tuning"],
                                        "kernel_ms_per_step": {k: v[0] / v[1] for k, v in fp32_only["kt"].items()}}
        line["speedup_vs_plain_fp64"] = pms / ms_step
        line["e2e_speedup_vs_plain_fp64"] = line["e2e"]["value"] / line["plain_fp64"]["e2e"]["value"]
        if world == 1 and args.error_study:
            line["error_vs_fp64"] = error_study(pkg, m, p, st, head["tuning"], closure)
    if world == 1 and args.large and args.nq != 192:
        line["large_shell"] = run_large(pkg, args, barrier, dev)
    if args.cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(args, m, p, st)
    return line


def run_large(pkg, args, barrier, dev):
    """The 6x192x192x40 shell (8,847,360 cells): the mixed step with MLP sources
    and the plain FP64 step, K steps each, same measurement as the headline."""
    import argparse as _ap

    a = _ap.Namespace(**vars(args))
    a.nq = 192
    m, p, st, _ = pkg.problems.heliosphere_shell(nq=192, nlayer=args.nlayer, move=True, flux_precision=32)
    C = m["cell_nodes"].shape[0]
    closure, _ = load_closure(pkg, m, st)
    mix = measure_mode(pkg, m, p, st, 32, closure, a, barrier, dev, e2e_steps=3)
    f64 = measure_mode(pkg, m, p, st, 64, None, a, barrier, dev, e2e_steps=3)
    out = {"workload": f"heliosphere shell 6x192x192x{args.nlayer} = {C} cells, ALE", "cells": C}
    for tag, r, net in (("mixed_mlp", mix, True), ("plain_fp64", f64, False)):
        ms = r["ms"] / args.steps
        out[tag] = {"value": C / (ms / 1e3), "ms_per_step": ms, "clocks": r["clocks"], "tuning": r["tuning"],
                    "e2e": {"value": C * r["e2e_steps"] / r["e2e_wall"], "unit": UNIT},
                    "step_roofline": step_roofline(m, True, net, ms, list(r["kt"])),
                    "kernel_ms_per_step": {k: v[0] / v[1] for k, v in r["kt"].items()}}
    out["speedup_vs_plain_fp64"] = out["plain_fp64"]["ms_per_step"] / out["mixed_mlp"]["ms_per_step"]
    out["coupled"] = run_coupled_loop(pkg, m, p, st, closure, args, barrier, dev)
    return out


COUPLED_STEPS, COUPLED_MC_EVERY = 300, 100
COUPLED_MC = dict(n_H=0.18, u_H=(-2.6, 0.0, 0.0), cp_H=float(np.sqrt(2.0 * (0.06 * 1.3 ** 2 / (5.0 / 3.0)) / 0.06)),
                  n_particles=10_000_000)


def run_coupled_loop(pkg, m, p, st, closure, args, barrier, dev, steps=COUPLED_STEPS):
    """The large configuration's coupled loop (closure.run_coupled): the mixed
    step with MLP sources every step and, every 100 steps, a Monte-Carlo pass
    (1e7 neutrals) through the current plasma whose sources the cells outside
    the closure's training envelope take; timed with CUDA events on the
    context's stream around the whole loop, passes included."""
    import torch

    C = m["cell_nodes"].shape[0]
    step, tuning = make_step(pkg, m, p, st, 32, args.tuning, closure)
    step.go(max(args.warmup, 3))
    stream = torch.cuda.ExternalStream(step.stream())
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(dev) as clk:
        ev0.record(stream)
        r = pkg.closure.run_coupled(step, closure, steps, mc_every=COUPLED_MC_EVERY, **COUPLED_MC)
        ev1.record(stream)
        barrier()
    ms = ev0.elapsed_time(ev1)
    step.close()
    return {"steps": steps, "mc_every": COUPLED_MC_EVERY, "mc_passes": r["mc_passes"],
            "mc_particles": COUPLED_MC["n_particles"], "value": C * steps / (ms / 1e3), "unit": UNIT,
            "ms_per_step": ms / steps, "clocks": clk.summary(),
            "cells_outside_envelope": r["outside_last_step"],
            "note": "device time of the whole loop, the Monte-Carlo passes and their fallback hand-over included"}


def timed_oracle(m, p, st, steps, warmup=1):
    """Seconds for `steps` oracle steps of the workload (after `warmup`), with
    the reference's own compiled Phys_param::chlld solving every face where
    oracle/_ref holds it (the Riemann solves are most of the step's host time;
    the results are identical to the oracle's restatement). Returns
    (seconds, threads, where the Riemann solver came from)."""
    import oracle_lib as ol

    run = ol.OracleRun(m, p)
    s = np.ascontiguousarray(st.copy())
    used_ref = ol.use_reference_riemann(p["gamma"])
    try:
        run.go(s, max(warmup, 1))  # first touch / geometry warm-up
        t0 = time.perf_counter()
        run.go(s, steps)
        dt = time.perf_counter() - t0
    finally:
        ol.use_reference_riemann(None)
    solver = ("the reference's own compiled Phys_param::chlld on every face" if used_ref
              else "the oracle's restatement of chlld (the reference's was not built)")
    return dt, int(ol.oracle().oracle_num_threads()), solver


def cpu_baseline(args, m, p, st, steps=None):
    """The oracle (OpenMP restatement of Setka::Go's plasma loop) on the same
    mesh, a bounded number of steps."""
    steps = steps or args.cpu_steps
    dt, cores, solver = timed_oracle(m, p, st, steps)
    C = m["cell_nodes"].shape[0]
    return {"value": C * steps / dt, "unit": UNIT, "cores": cores,
            "kind": "port", "sample": f"{steps} steps of the full {C}-cell workload "
                                      f"({dt:.1f} s), oracle/titan_oracle.cpp with OpenMP, {solver}"}


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
    stream = torch.cuda.ExternalStream(plasma.stream())  # the loop runs on the context's stream
    barrier()
    with ClockSampler(dev) as clk:
        ev0.record(stream)
        ss.go(args.steps)
        ev1.record(stream)
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
    dt, cores, solver = timed_oracle(m, p, st, args.steps, args.warmup)
    v = C * args.steps / dt
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded heliosphere-like shell)",
            "config": {"workload": f"heliosphere shell 6x{args.nq}x{args.nq}x{args.nlayer} = {C} cells, ALE, "
                                   "HLLD/HLLC, FP64", "cells": C},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{args.steps} steps of the full workload after {args.warmup} warm-up, "
                                       f"oracle/titan_oracle.cpp with OpenMP, {solver}"},
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
    ap.add_argument("--cpu-steps", type=int, default=30)
    ap.add_argument("--tuning", default="auto", help="auto, or 'face_variant,cell_variant'")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-large", dest="large", action="store_false",
                    help="skip the 6x192x192x40 shell sub-run (mixed + plain FP64)")
    ap.add_argument("--shard", action="store_true",
                    help="split one mesh over the GPUs (strong scaling) instead of N replicas")
    args = ap.parse_args()
    if args.impl == "reference":
        # a bounded sample of the workload: a full step takes about 0.12-0.2 s
        # on 16 host threads, so up to 100 steps (the line states the count it ran)
        args.steps = min(args.steps, 100)
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
