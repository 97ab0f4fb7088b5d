"""The bench line's roofline arithmetic, checked on the CPU against the
hot-path scope's own figures: the algorithmic bytes per cell-update of the
step (305 / 308.5 B on a stationary mesh, 362.4 B with node motion on the
heliosphere shell, 36 B more with the closure), the network's 101,632 FLOP per
cell, and the captured DRAM traffic per step over those bytes (2.9x for the
FP64 step, 3.04x for the mixed step on the 6x96x96x40 shell)."""
import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    argv = sys.argv
    try:
        sys.argv = ["bench.py"]
        spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        sys.argv = argv
    return mod


def _counts(C, F, N):
    """A mesh dict with only the row counts the accounting reads (no memory)."""
    z = np.zeros((), dtype=np.int8)
    return {"cell_nodes": np.broadcast_to(z, (C, 8)), "face_nodes": np.broadcast_to(z, (F, 4)),
            "node_xyz": np.broadcast_to(z, (N, 3))}


SHELL96 = _counts(2211840, 6690816, 2267218)     # 6x96x96x40: (6*96^2+2)*41 nodes
SHELL192 = _counts(8847360, 26763264, 9068626)   # 6x192x192x40: (6*192^2+2)*41 nodes
CUBE32 = _counts(32768, 101376, 35937)


def test_step_bytes_per_cell_update(bench):
    _, b = bench.step_bytes(CUBE32, move=False, closure=False)
    assert b == pytest.approx(136 + 24 + 48 * 101376 / 32768) and round(b, 1) == 308.5
    _, b = bench.step_bytes(SHELL96, move=False, closure=False)
    assert round(b, 1) == 305.2
    total, b = bench.step_bytes(SHELL96, move=True, closure=False)
    assert round(b, 1) == 362.4 and total == pytest.approx(801574752.0)
    total, b = bench.step_bytes(SHELL96, move=True, closure=True)
    assert round(b, 1) == 398.4 and total == pytest.approx(881200992.0)


def test_closure_flop_per_cell(bench):
    bound, flop = bench.kernel_work("closure_mlp", SHELL96, move=True, sources=True)
    assert bound == "tensor" and flop == 2211840 * 101632


def test_captured_traffic_over_algorithmic_bytes(bench):
    mixed = ["move_nodes", "closure_mlp", "face_flux_fp32", "cell_update"]
    fp64 = ["move_nodes", "face_flux_fp64", "cell_update"]
    for mesh, C, lo, hi in ((SHELL96, 2211840, 2.8, 3.1), (SHELL192, 8847360, 2.9, 3.25)):
        for kernels, closure in ((mixed, True), (fp64, False)):
            tr = [bench.traffic(k, C, closure) for k in kernels]
            assert all(t is not None for t in tr)
            total, _ = bench.step_bytes(mesh, move=True, closure=closure)
            assert lo < sum(tr) / total < hi
    assert bench.traffic("cell_update", 1000, False) is None   # other sizes report none


def test_step_roofline_is_bytes_over_time(bench):
    r = bench.step_roofline(SHELL96, True, False, 1.0, ["move_nodes", "face_flux_fp64", "cell_update"])
    assert r["achieved"] == pytest.approx(801574752.0 / 1e-3 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    assert r["traffic_over_algorithmic"] == pytest.approx(r["traffic_per_step"] / r["algorithmic_bytes_per_step"])


def test_reference_arm_line_on_a_small_shell(bench, oracle_lib):
    """`bench.py --impl reference` on a small shell: the oracle times its FP64
    step on the host and prints the line the driver reads (rank 0 only)."""
    import argparse
    args = argparse.Namespace(nq=6, nlayer=6, mode="mixed-mlp", steps=2, warmup=1)
    line = bench.run_reference(args, 0, 1)
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "cell-updates/s"
    assert line["config"]["cells"] == 6 * 6 * 6 * 6
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert bench.run_reference(args, 1, 2) is None   # other ranks do no work


def test_cpu_timing_names_the_riemann_solver_it_ran(bench, oracle_lib, titan, monkeypatch):
    """The CPU baseline uses the reference's compiled solver where oracle/_ref
    holds it and says so; without it, the oracle's restatement, also said."""
    import oracle_lib as ol
    m, p, st, _ = titan.problems.heliosphere_shell(nq=6, nlayer=6, move=True)
    dt, cores, solver = bench.timed_oracle(m, p, st, 1)
    assert dt > 0 and cores >= 1
    assert ("reference's own compiled" in solver) == ol.ref_available()
    monkeypatch.setattr(ol, "ref_available", lambda: False)
    _, _, solver = bench.timed_oracle(m, p, st, 1)
    assert "restatement" in solver
