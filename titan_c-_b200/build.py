"""Builds libtitan_b200.so in-tree with nvcc for sm_100a.

    python titan_c-_b200/build.py [--force]

Translation units and their floating-point flags:
  kernels_fp64.cu  -fmad=false  geometry, FP64 flux, cell update (bit-exact FP64)
  kernels_fp32.cu  -fmad=true -prec-div=false -prec-sqrt=false
                                FP32 Riemann flux of the mixed-precision step
  kernels_tvd_fp64.cu, kernels_tvd_fp32.cu   the same with second-order faces
  kernels_cell.cu  -fmad=false  cell update (gather, update, sources, floors, next-layer geometry)
  surface.cu       -fmad=false  surface-tracking node motion (TS / HP / BS speeds, rays)
  halo.cu                       whole-cell copies for the halo exchange of a sharded step
  mc_neutral.cu                 Monte-Carlo neutral hydrogen (source generator)
  closure_mlp.cu                closure inference on tcgen05 / TMEM (per step)
  closure_train.cu, closure_api.cu   closure training (BF16 tensor-core GEMMs), C ABI
  titan_api.cu, renumber.cpp    host side of the C ABI
  checkpoint.cpp                cell-parameter files in the reference's layout
  noalloc.cu       -fmad=false  titan_step_noalloc (fixed scratch array, no allocation)

It also builds tests/cpp/setka_consumer.cpp (g++, host only) into _build/: a
C++ program that drives the library through include/titan_b200.h the way the
binding inside the reference's Setka does (used by the GPU tests).
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtitan_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "--expt-relaxed-constexpr"]

UNITS = [
    ("kernels_fp64.cu", ["-fmad=false"]),
    ("kernels_fp32.cu", ["-fmad=true", "-prec-div=false", "-prec-sqrt=false"]),
    ("kernels_tvd_fp64.cu", ["-fmad=false"]),
    ("kernels_cell.cu", ["-fmad=false"]),
    ("surface.cu", ["-fmad=false"]),
    ("halo.cu", []),
    ("kernels_tvd_fp32.cu", ["-fmad=true", "-prec-div=false", "-prec-sqrt=false"]),
    ("mc_neutral.cu", []),
    ("closure_mlp.cu", []),
    ("closure_train.cu", []),
    ("closure_api.cu", []),
    ("titan_api.cu", []),
    ("noalloc.cu", ["-fmad=false"]),
    ("renumber.cpp", []),
    ("checkpoint.cpp", []),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _includes(path: str, seen: set[str]) -> set[str]:
    """Local headers `path` includes (#include "..."), transitively."""
    for line in open(path, errors="replace"):
        m = re.match(r'\s*#\s*include\s+"([^"]+)"', line)
        if m:
            h = os.path.normpath(os.path.join(os.path.dirname(path), m.group(1)))
            if os.path.exists(h) and h not in seen:
                seen.add(h)
                _includes(h, seen)
    return seen


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    """Compiles the stale translation units in parallel and links the library."""
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(BUILD, exist_ok=True)
    objs, cmds = [], []
    for src, flags in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s, __file__] + sorted(_includes(s, set()))):
            cmd = [nvcc(), *ARCH, *COMMON, *flags, *(extra or []), "-c", s, "-o", o]
            if src.endswith(".cpp"):
                cmd = [nvcc(), *COMMON, "-Wno-deprecated-gpu-targets", "-x", "c++", "-c", s, "-o", o]
            cmds.append(cmd)
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd), flush=True)
    workers = max(1, min(len(cmds), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as pool:
        for r in list(pool.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds)):
            if r.stdout or r.stderr:
                print(r.stdout + r.stderr, end="", flush=True)
            r.check_returncode()
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    build_consumer(force, verbose)
    return LIB


CONSUMER_SRC = os.path.join(os.path.dirname(HERE), "tests", "cpp", "setka_consumer.cpp")
CONSUMER = os.path.join(BUILD, "setka_consumer")


def build_consumer(force: bool = False, verbose: bool = False) -> str | None:
    """The C++ consumer of the ABI, linked against the in-tree library (rpath
    relative to the binary, so the tree can move)."""
    if not os.path.exists(CONSUMER_SRC):
        return None
    inc = os.path.join(os.path.dirname(HERE), "include")
    if force or _stale(CONSUMER, [CONSUMER_SRC, LIB, os.path.join(inc, "titan_b200.h")]):
        cxx = shutil.which("g++") or "g++"
        cmd = [cxx, "-O2", "-std=c++17", f"-I{inc}", CONSUMER_SRC, "-o", CONSUMER, f"-L{HERE}", "-ltitan_b200",
               "-Wl,-rpath,$ORIGIN/.."]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return CONSUMER


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
    print(LIB)
