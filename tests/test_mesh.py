"""Synthetic meshes: counts of the benchmark configurations and the geometry
invariants of Setka::Test_geometr (TITAN/source/Setka.cpp:467-620)."""
import numpy as np
import pytest

import oracle_lib as ol


def _invariants(mesh, geom, closure=1e-12):
    fc = mesh["face_cells"]
    cc = geom["cell_center"]
    n = geom["face_normal"]
    # Test 1: a face has one or two cells; the normal points from cells[0] to cells[1]
    assert np.all(fc[:, 0] >= 0)
    two = fc[:, 1] >= 0
    d = cc[fc[two, 1]] - cc[fc[two, 0]]
    assert np.all(np.sum(n[two] * d, axis=1) > 0.0)
    # Test 2: 6 faces and 8 nodes per cell (structural)
    assert mesh["cell_faces"].shape[1] == 6 and mesh["cell_nodes"].shape[1] == 8
    # every cell is listed by each of its faces
    C = mesh["cell_faces"].shape[0]
    own = fc[mesh["cell_faces"]]
    assert np.all((own[:, :, 0] == np.arange(C)[:, None]) | (own[:, :, 1] == np.arange(C)[:, None]))
    # Test 5: unit normals and closed cells (sum of signed n*A vanishes)
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-14)
    sign = np.where(own[:, :, 0] == np.arange(C)[:, None], 1.0, -1.0)
    s = np.einsum("cs,csk->ck", sign * geom["face_area"][mesh["cell_faces"]], n[mesh["cell_faces"]])
    scale = geom["face_area"][mesh["cell_faces"]].max(axis=1)
    # exact for planar faces; the spherical quads of a coarse shell are slightly warped
    assert np.all(np.linalg.norm(s, axis=1) <= closure * scale)


def test_cube_counts(titan):
    m = titan.mesh.cube_mesh(32)
    assert m["cell_nodes"].shape == (32768, 8)
    assert m["face_nodes"].shape == (101376, 4)
    assert int((m["face_cells"][:, 1] < 0).sum()) == 6144
    assert m["node_xyz"].shape == (35937, 3)


def test_shell_counts_formula(titan):
    nq, nl = 6, 5
    m = titan.mesh.shell_mesh(nq, nl)
    assert m["cell_nodes"].shape[0] == 6 * nq * nq * nl
    assert m["node_xyz"].shape[0] == (6 * nq * nq + 2) * (nl + 1)
    assert m["face_nodes"].shape[0] == 6 * nq * nq * (nl + 1) + 12 * nq * nq * nl
    ft = m["face_type"]
    assert int((ft == 1).sum()) == 6 * nq * nq
    assert int(((ft == 2) | (ft == 3)).sum()) == 6 * nq * nq


def test_cube_geometry_invariants(titan, oracle_lib):
    m = titan.mesh.cube_mesh(8)
    run = ol.OracleRun(m, titan.problems.params())
    g = run.geometry()
    _invariants(m, g)
    assert abs(g["cell_volume"].sum() - 1.0) < 1e-12
    assert np.allclose(g["face_area"], 1.0 / 64)


@pytest.mark.parametrize("dims", [(1, 1, 1), (1, 40, 1), (3, 1, 2), (5, 7, 3), (33, 2, 5)])
def test_ragged_box_counts_and_invariants(titan, oracle_lib, dims):
    """The boxes of the size and shape edge cases: counts, the invariants
    above, and volumes and areas of the unit box cut nx x ny x nz."""
    nx, ny, nz = dims
    m = titan.mesh.box_mesh(nx, ny, nz)
    assert m["cell_nodes"].shape[0] == nx * ny * nz
    assert m["node_xyz"].shape[0] == (nx + 1) * (ny + 1) * (nz + 1)
    assert m["face_nodes"].shape[0] == (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1)
    assert int((m["face_cells"][:, 1] < 0).sum()) == 2 * (ny * nz + nx * nz + nx * ny)
    g = ol.OracleRun(m, titan.problems.params()).geometry()
    _invariants(m, g)
    assert abs(g["cell_volume"].sum() - 1.0) < 1e-12
    assert np.allclose(g["cell_volume"], 1.0 / (nx * ny * nz), rtol=1e-12)
    n = np.abs(g["face_normal"])
    for axis, area in ((0, 1.0 / (ny * nz)), (1, 1.0 / (nx * nz)), (2, 1.0 / (nx * ny))):
        along = n[:, axis] > 0.5
        assert int(along.sum()) == ((nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1))[axis]
        assert np.allclose(g["face_area"][along], area, rtol=1e-12)


def test_shell_geometry_invariants(titan, oracle_lib):
    m = titan.mesh.shell_mesh(6, 5)
    run = ol.OracleRun(m, titan.problems.params())
    g = run.geometry()
    _invariants(m, g, closure=5e-3)
    vol = g["cell_volume"].sum()
    exact = 4.0 / 3.0 * np.pi * (100.0 ** 3 - 1.0)
    assert 0.85 * exact < vol < exact
    assert np.all(g["cell_volume"] > 0)


def test_oracle_geometry_matches_numpy(titan, oracle_lib):
    m = titan.mesh.shell_mesh(4, 3)
    run = ol.OracleRun(m, titan.problems.params())
    g = run.geometry()
    cc, fc, nrm, area = titan.mesh.hex_geometry(m)
    np.testing.assert_allclose(g["cell_center"], cc, rtol=0, atol=1e-12)
    np.testing.assert_allclose(g["face_center"], fc, rtol=0, atol=1e-12)
    np.testing.assert_allclose(g["face_normal"], nrm, rtol=0, atol=1e-12)
    np.testing.assert_allclose(g["face_area"], area, rtol=1e-12)


def test_face_builder_first_proposer_keeps_order(titan):
    m = titan.mesh.cube_mesh(2)
    cn, fnd, fcl, cf = m["cell_nodes"], m["face_nodes"], m["face_cells"], m["cell_faces"]
    hexf = titan.mesh.HEX_FACES
    for c in range(cn.shape[0]):
        for s in range(6):
            f = cf[c, s]
            quad = cn[c, hexf[s]]
            assert set(quad) == set(fnd[f])
            if fcl[f, 0] == c:
                np.testing.assert_array_equal(fnd[f], quad)


@pytest.mark.parametrize("n", [1, 3])
def test_small_cubes_build(titan, n):
    m = titan.mesh.cube_mesh(n)
    assert m["face_nodes"].shape[0] == 3 * n * n * (n + 1)
