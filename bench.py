"""Benchmark of the B200 plasma step: MHD cell-updates/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--nq 96] [--nlayer 40] [--flux 64|32]

Workload (N=1): the heliosphere-like shell — cubed sphere 6x96x96 x 40
geometric layers = 2,211,840 hexahedra, r in [1, 100], supersonic Parker-spiral
wind inside, interstellar inflow outside, seeded lognormal perturbation,
HLLD where B^2/(8 pi p) > 0.01 else HLLC, prescribed radial node motion (ALE),
all-FP64. One step = one pass of the plasma loop over every face and cell.

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
                                                 flux_precision=args.flux)
    return pkg, m, p, st


def face_flux_bytes(m, move: bool, fp32: bool) -> float:
    """Algorithmic DRAM bytes of one face-flux launch: every input read once,
    every output written once (kernel K2)."""
    C = m["cell_nodes"].shape[0]
    F = m["face_nodes"].shape[0]
    N = m["node_xyz"].shape[0]
    per_face = 8 + 2 + 3 * 8 + 8 + 8      # c0,c1 | type,method | normal | area | half distance
    state = 8 * 8 * C                       # 8 FP64 primitives per cell, read once
    out = (9 * (4 if fp32 else 8)) * F      # 9 fluxes (x area) per face
    # moving mesh: face node ids + node coordinates of both layers replace the
    # stored normal / area / half distance, and cell centres are read instead
    ale = (16 * F + 2 * 24 * N + 24 * C - 40 * F) if move else 0
    return float(per_face * F + state + out + ale)


def run_ours(args, rank, world):
    import torch

    dev = rank % max(torch.cuda.device_count(), 1)
    torch.cuda.set_device(dev)
    pkg, m, p, st = build_problem(args)
    C = m["cell_nodes"].shape[0]
    F = m["face_nodes"].shape[0]
    step = pkg.PlasmaStep(m, p)
    step.upload_state(st)
    if args.tuning == "auto":
        tuning = step.autotune(reps=3)
    else:
        fv, cv = (int(x) for x in args.tuning.split(","))
        step.set_tuning(fv, cv)
        tuning = step.tuning()
    kernels_per_step = 3 if p["move"] else 2
    flux_name = "face_flux_fp32" if args.flux == 32 else "face_flux_fp64"

    # warm-up (also captures the CUDA graph)
    step.go(max(args.warmup, 3))
    stream = torch.cuda.ExternalStream(step.stream())
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    barrier()
    with ClockSampler(dev) as clk:
        ev0.record(stream)
        step.go(args.steps)
        ev1.record(stream)
        barrier()
    ms = ev0.elapsed_time(ev1)
    clocks = clk.summary()

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
    ev0.record(stream)
    for _ in range(e2e_steps):
        step.upload_state(host)
        step.go(1)
        step.download_state(host)
    ev1.record(stream)
    barrier()
    e2e_wall = time.perf_counter() - t0
    ns = 8 + p["npassive"]
    step.close()

    t = torch.tensor([ms, e2e_wall], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms, e2e_wall = float(t[0]), float(t[1])
    if rank != 0:
        return None
    value = world * C * args.steps / (ms / 1e3)
    hbm, src = peaks()
    bytes_launch = face_flux_bytes(m, bool(p["move"]), args.flux == 32)
    achieved = bytes_launch / (k_avg / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.flux == 64 else "f32-flux/f64-update",
        "data": "synthetic (seeded heliosphere-like shell; no external data)",
        "config": {"workload": f"heliosphere shell 6x{args.nq}x{args.nq}x{args.nlayer} = {C} cells, {F} faces, "
                               f"ALE, HLLD/HLLC, FP{args.flux} flux", "cells": C, "faces": F,
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU", "tuning": tuning,
                   "l2": "inputs larger than L2 (state 141 MB + face data 0.5 GB), no flush"},
        "face_fluxes_per_s": world * F * args.steps / (ms / 1e3),
        "e2e": {"value": world * C * e2e_steps / e2e_wall, "unit": UNIT,
                "h2d_bytes_per_step": 8 * ns * C, "d2h_bytes_per_step": 8 * ns * C},
        "gpu_launches": args.steps * kernels_per_step,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "kernel": flux_name, "peak_source": src,
                     "algorithmic_bytes_per_launch": bytes_launch, "avg_launch_ms": k_avg,
                     "kernel_share": k_ms / total_k},
        "kernel_ms_per_step": {k: v[0] / v[1] for k, v in kt.items()},
        "clocks": clocks,
    }
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
    ap.add_argument("--flux", type=int, default=64, choices=[64, 32])
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--tuning", default="auto", help="auto, or 'face_variant,cell_variant'")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    args = ap.parse_args()
    if args.impl == "reference":
        args.steps = min(args.steps, 3)
        args.warmup = min(args.warmup, 1)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and args.impl == "ours":
        import torch
        import datetime

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", rank)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    line = run_reference(args, rank, world) if args.impl == "reference" else run_ours(args, rank, world)
    if world > 1 and args.impl == "ours":
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
