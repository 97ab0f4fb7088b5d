"""The drop-in boundary from C++: a program that includes include/titan_b200.h,
holds the mesh as the reference's Setka object graph (Yzel / Gran / Cell with
1-based `number` and per-cell parameter maps), flattens it as the binding in
INTEGRATION.md does (Setka::Gpu_init), steps it through titan_step in two
Go-like calls (Setka::Go, TITAN/source/Setka.h:221) and writes its mesh and
states (tests/cpp/setka_consumer.cpp, compiled by the library build). The
oracle steps the same flattened mesh; every cell's state, dt and t must agree
within 1e-12 relative (the FP64 step is bit-exact against the oracle)."""
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu


def _read(path):
    with open(path, "rb") as f:
        N, C, F, steps = np.fromfile(f, dtype=np.int64, count=4)
        xyz = np.fromfile(f, dtype=np.float64, count=3 * N).reshape(N, 3)
        cn = np.fromfile(f, dtype=np.int32, count=8 * C).reshape(C, 8)
        cf = np.fromfile(f, dtype=np.int32, count=6 * C).reshape(C, 6)
        fn = np.fromfile(f, dtype=np.int32, count=4 * F).reshape(F, 4)
        fc = np.fromfile(f, dtype=np.int32, count=2 * F).reshape(F, 2)
        ft = np.fromfile(f, dtype=np.int8, count=F)
        s0 = np.fromfile(f, dtype=np.float64, count=10 * C).reshape(10, C)
        s1 = np.fromfile(f, dtype=np.float64, count=10 * C).reshape(10, C)
        dt, t = np.fromfile(f, dtype=np.float64, count=2)
    mesh = dict(node_xyz=xyz, cell_nodes=cn, cell_faces=cf, cell_type=np.zeros(C, np.int8),
                cell_tvd=np.ones(C, np.uint8), face_nodes=fn, face_cells=fc, face_type=ft,
                face_surf=np.zeros(F, np.int8), face_bc=np.full(F, -1, np.int32), bc_vals=np.zeros((0, 10)),
                node_amp=None, node_phase=None)
    return mesh, int(steps), s0, s1, float(dt), float(t)


def test_cpp_setka_binding_matches_oracle(titan, built_lib, oracle_lib, tmp_path):
    build = __import__("importlib").import_module("titan_c-_b200.build")
    exe = build.build_consumer()
    assert exe and os.path.exists(exe)
    out = tmp_path / "consumer.bin"
    r = subprocess.run([exe, "12", "20", str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    mesh, steps, s0, s1, dt, t = _read(out)
    # the C++ program built the same cube as the Python mesh builder (New_connect order)
    ref_mesh = titan.mesh.cube_mesh(12)
    for k in ("cell_nodes", "cell_faces", "face_nodes", "face_cells"):
        np.testing.assert_array_equal(mesh[k], ref_mesh[k])
    p = titan.problems.params(KFL=0.4, soft_fixups=0, method_policy=0)
    run = ol.OracleRun(mesh, p)
    run.set_face_method(np.full(mesh["face_nodes"].shape[0], 3, dtype=np.int8))
    ref = np.ascontiguousarray(s0.copy())
    run.go(ref, steps)
    scale = np.maximum(np.abs(ref[:8]), 1e-12 * np.abs(ref[:8]).max())
    assert float(np.max(np.abs(s1[:8] - ref[:8]) / scale)) <= 1e-12
    assert abs(dt - run.clock[0]) <= 1e-12 * run.clock[0]
    assert abs(t - run.clock[1]) <= 1e-12 * max(run.clock[1], 1e-300)
