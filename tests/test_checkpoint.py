"""Cell-parameter checkpoints in the reference's binary layout
(Setka::Save_cell_parameters / Download_cell_parameters,
TITAN/source/Setka_physics.cpp:4108-4231), through the library's host-only
C ABI. `reference_layout_bytes` restates the reference writer's layout (the
reference's mesh driver cannot be built here) to produce files as TITAN
writes them: keys in an arbitrary order, keys this library does not carry,
the node block, and the 1000 reserved bools."""
import ctypes
import os
import struct

import numpy as np
import pytest

NAMES = ["rho", "Vx", "Vy", "Vz", "p", "Bx", "By", "Bz", "Q", "rho_He"]


def reference_layout_bytes(cells: list, nodes=None) -> bytes:
    """cells: list of dicts key -> value, in the order the writer meets them."""
    out = bytearray()
    for d in cells:
        out += struct.pack("<Q", len(d))
        for k, v in d.items():
            kb = k.encode()
            out += struct.pack("<Q", len(kb)) + kb + struct.pack("<d", v)
    out += struct.pack("<?", nodes is not None)
    if nodes is not None:
        out += struct.pack("<Q", len(nodes))
        out += np.ascontiguousarray(nodes, dtype="<f8").tobytes()
    out += b"\x00" * 1000
    return bytes(out)


def _read(N, path, ncell, nnode, init=None):
    st = np.zeros((10, ncell)) if init is None else np.ascontiguousarray(init.copy())
    xyz = np.zeros((nnode, 3))
    found, has = ctypes.c_int32(0), ctypes.c_int32(0)
    rc = N.lib().titan_read_cell_parameters(str(path).encode(), ncell, nnode, N.ptr(st), N.ptr(xyz),
                                            ctypes.byref(found), ctypes.byref(has))
    return rc, st, xyz, found.value, has.value


def test_write_then_read_is_bitexact(built_lib, titan, tmp_path):
    N = titan.native
    rng = np.random.default_rng(0)
    C, V = 57, 91
    st = np.ascontiguousarray(rng.standard_normal((10, C)))
    xyz = np.ascontiguousarray(rng.standard_normal((V, 3)))
    path = tmp_path / "parameters_0001.bin"
    N.check(N.lib().titan_write_cell_parameters(str(path).encode(), C, 10, N.ptr(st), V, N.ptr(xyz)))
    rc, back, bx, found, has = _read(N, path, C, V)
    assert rc == 0 and has == 1 and found == (1 << 10) - 1
    assert np.array_equal(back.view(np.uint64), st.view(np.uint64))
    assert np.array_equal(bx.view(np.uint64), xyz.view(np.uint64))
    # the writer's bytes are the reference layout with keys in field order
    cells = [{k: st[i, c] for i, k in enumerate(NAMES)} for c in range(C)]
    assert path.read_bytes() == reference_layout_bytes(cells, xyz)


def test_reads_a_reference_file_with_foreign_keys_in_any_order(built_lib, titan, tmp_path):
    N = titan.native
    rng = np.random.default_rng(1)
    C, V = 40, 12
    truth = rng.standard_normal((10, C))
    cells = []
    for c in range(C):
        d = {k: truth[i, c] for i, k in enumerate(NAMES[:8])}           # no passive scalars in this file
        d.update({"rho_H1": 0.18, "Vx_H4": -2.5, "p_Pui_1": 1e-3, "n_H4_MK": 7.0})
        keys = list(d)
        rng.shuffle(keys)
        cells.append({k: d[k] for k in keys})
    nodes = rng.standard_normal((V, 3))
    path = tmp_path / "parameters_0216.bin"
    path.write_bytes(reference_layout_bytes(cells, nodes))
    init = np.full((10, C), 123.0)
    rc, st, xyz, found, has = _read(N, path, C, V, init)
    assert rc == 0 and has == 1
    assert found == (1 << 8) - 1
    assert np.array_equal(st[:8], truth[:8])
    assert (st[8:] == 123.0).all()            # absent keys keep the caller's values
    assert np.array_equal(xyz, nodes)


def test_file_without_node_block_and_errors(built_lib, titan, tmp_path):
    N = titan.native
    cells = [{"rho": 1.0 + c, "p": 2.0} for c in range(5)]
    p1 = tmp_path / "a.bin"
    p1.write_bytes(reference_layout_bytes(cells, None))
    rc, st, _, found, has = _read(N, p1, 5, 3)
    assert rc == 0 and has == 0 and found == (1 << 0) | (1 << 4)
    assert list(st[0]) == [1.0, 2.0, 3.0, 4.0, 5.0]
    # node count that does not match the mesh
    p2 = tmp_path / "b.bin"
    p2.write_bytes(reference_layout_bytes(cells, np.zeros((4, 3))))
    rc, *_ = _read(N, p2, 5, 3)
    assert rc == -2  # TITAN_EMESH
    assert b"nodes" in N.lib().titan_last_error()
    # a truncated file
    p3 = tmp_path / "c.bin"
    p3.write_bytes(reference_layout_bytes(cells, None)[:40])
    rc, *_ = _read(N, p3, 5, 3)
    assert rc != 0
    assert b"truncated" in N.lib().titan_last_error() or b"malformed" in N.lib().titan_last_error()
    # a missing file
    rc, *_ = _read(N, tmp_path / "missing.bin", 5, 3)
    assert rc != 0
