"""The C ABI library: it loads, exports every declared symbol, and its host-only
logic (validation, SFC renumbering) behaves — no device call is made here."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "titan_b200.h")


def declared_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(titan_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_the_boundary():
    syms = declared_symbols()
    for s in ["titan_create", "titan_step", "titan_upload_state", "titan_download_state", "titan_destroy",
              "titan_riemann_batch", "titan_set_face_method", "titan_set_sources"]:
        assert s in syms


def test_library_exports_every_declared_symbol(built_lib, titan):
    for s in declared_symbols():
        assert hasattr(built_lib, s), s
        assert s in titan.native.SIGNATURES, s


def test_version_and_error_string(built_lib):
    assert b"sm_100a" in built_lib.titan_version()
    assert isinstance(built_lib.titan_last_error(), bytes)


def _renumber(titan, m):
    N = titan.native
    C, F, V = m["cell_nodes"].shape[0], m["face_nodes"].shape[0], m["node_xyz"].shape[0]
    c = np.empty(C, np.int32)
    f = np.empty(F, np.int32)
    n = np.empty(V, np.int32)
    rc = N.lib().titan_sfc_renumber(V, C, F, N.ptr(m["node_xyz"]), N.ptr(m["cell_nodes"], N.I32),
                                    N.ptr(m["face_cells"], N.I32), N.ptr(c, N.I32), N.ptr(f, N.I32),
                                    N.ptr(n, N.I32))
    N.check(rc)
    return c, f, n


def test_sfc_renumbering_is_a_bitexact_permutation(built_lib, titan):
    m = titan.mesh.shell_mesh(6, 4)
    c, f, n = _renumber(titan, m)
    for p, size in [(c, m["cell_nodes"].shape[0]), (f, m["face_nodes"].shape[0]), (n, m["node_xyz"].shape[0])]:
        assert np.array_equal(np.sort(p), np.arange(size))
    # round trip of a state through the permutation and its inverse is bit-exact
    rng = np.random.default_rng(0)
    st = rng.standard_normal((10, len(c)))
    fwd = st[:, c]
    back = np.empty_like(fwd)
    back[:, c] = fwd
    assert np.array_equal(back.view(np.uint64), st.view(np.uint64))
    # faces follow the new index of their cells[0]
    inv = np.empty_like(c)
    inv[c] = np.arange(len(c))
    owner_new = inv[m["face_cells"][f, 0]]
    assert np.all(np.diff(owner_new) >= 0)


def test_sfc_renumbering_improves_locality(built_lib, titan):
    m = titan.mesh.shell_mesh(12, 8)
    c, f, n = _renumber(titan, m)
    inv = np.empty_like(c)
    inv[c] = np.arange(len(c))
    fc = m["face_cells"]
    inner = fc[:, 1] >= 0
    before = np.median(np.abs(fc[inner, 0] - fc[inner, 1]))
    after = np.median(np.abs(inv[fc[inner, 0]] - inv[fc[inner, 1]]))
    assert after < before


def test_sfc_renumber_rejects_bad_index(built_lib, titan):
    m = titan.mesh.cube_mesh(2)
    cn = m["cell_nodes"].copy()
    cn[0, 0] = 10 ** 6
    m = dict(m, cell_nodes=cn)
    with pytest.raises(titan.TitanError) as e:
        _renumber(titan, m)
    assert e.value.code == -2


def test_create_rejects_inconsistent_mesh_before_touching_the_device(built_lib, titan):
    m, p, st, meth = titan.problems.brio_wu_cube(4)
    fc = m["face_cells"].copy()
    inner = np.nonzero(fc[:, 1] >= 0)[0][0]
    fc[inner, 1] = -1   # an interior face that lost its second cell
    bad = dict(m, face_cells=fc)
    with pytest.raises(titan.TitanError) as e:
        titan.PlasmaStep(bad, p)
    assert e.value.code == -2
    ft = m["face_type"].copy()
    ft[np.nonzero(m["face_cells"][:, 1] < 0)[0][0]] = 1   # hard face without fixed values
    with pytest.raises(titan.TitanError) as e:
        titan.PlasmaStep(dict(m, face_type=ft), p)
    assert e.value.code == -2
    with pytest.raises(titan.TitanError) as e:
        titan.PlasmaStep(m, dict(p, npassive=1))
    assert e.value.code == -2


def test_create_rejects_an_empty_mesh(built_lib, titan):
    m, p, _, _ = titan.problems.brio_wu_box(1, 1, 1)
    no_cells = dict(m, **{k: m[k][:0] for k in ("cell_nodes", "cell_faces", "cell_type", "cell_tvd")})
    no_faces = dict(m, **{k: m[k][:0] for k in ("face_nodes", "face_cells", "face_type", "face_surf", "face_bc")})
    for bad in (no_cells, no_faces, dict(m, node_xyz=m["node_xyz"][:0])):
        with pytest.raises(titan.TitanError) as e:
            titan.PlasmaStep(bad, p)
        assert e.value.code == -2 and "empty" in str(e.value)


def test_riemann_batch_argument_checks(built_lib, titan):
    N = titan.native
    rc = N.lib().titan_riemann_batch(0, None, None, None, None, None, 0, 64, 5.0 / 3.0, None, None, None)
    assert rc == 0
    rc = N.lib().titan_riemann_batch(4, None, None, None, None, None, 0, 64, 5.0 / 3.0, None, None, None)
    assert rc == -1
    one = np.zeros(8)
    rc = N.lib().titan_riemann_batch(1, N.ptr(np.zeros(1, np.int8), N.I8), N.ptr(np.zeros(3)), N.ptr(np.zeros(1)),
                                     N.ptr(one), N.ptr(one), 0, 16, 5.0 / 3.0, N.ptr(one), N.ptr(np.zeros(3)),
                                     N.ptr(np.zeros(1, np.int32), N.I32))
    assert rc == -1
