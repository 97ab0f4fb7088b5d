"""Synthetic hexahedral meshes in TITAN's cell / face / node conventions.

A mesh is a dict of numpy arrays matching ``titan_mesh`` (include/titan_b200.h):
node_xyz [N,3], cell_nodes [C,8], cell_faces [C,6], cell_type [C], cell_tvd [C],
face_nodes [F,4], face_cells [F,2], face_type [F], face_surf [F], face_bc [F],
bc_vals [B,10], and optionally node_amp / node_phase [N] for the prescribed
node motion.

Faces are built the way Setka::New_connect does (TITAN/source/Setka.cpp:2066-2130):
every cell proposes its six quads in the order (0,3,2,1), (4,5,6,7),
(0,1,5,4), (2,3,7,6), (1,2,6,5), (0,4,7,3); duplicates are merged, the first
proposer becomes cells[0] and keeps its node order, and each cell's six face
slots keep that proposal order (the order the flux gather runs in).
"""
from __future__ import annotations

import numpy as np

# node slots of the six faces of a hex, in the reference's order
HEX_FACES = np.array([[0, 3, 2, 1], [4, 5, 6, 7], [0, 1, 5, 4], [2, 3, 7, 6], [1, 2, 6, 5], [0, 4, 7, 3]],
                     dtype=np.int64)

_HASH_MUL = np.array([0x9E3779B97F4A7C15, 0xC2B2AE3D27D4EB4F, 0x165667B19E3779F9, 0x27D4EB2F165667C5],
                     dtype=np.uint64)


def build_faces(cell_nodes: np.ndarray):
    """Faces of a hexahedral mesh: (face_nodes [F,4], face_cells [F,2], cell_faces [C,6])."""
    cell_nodes = np.asarray(cell_nodes, dtype=np.int64)
    ncell = cell_nodes.shape[0]
    cand = cell_nodes[:, HEX_FACES].reshape(-1, 4)           # [6C, 4] in (cell, slot) order
    srt = np.sort(cand, axis=1).astype(np.uint64)
    with np.errstate(over="ignore"):
        h = srt[:, 0] * _HASH_MUL[0]
        for k in range(1, 4):
            h = (h ^ (h >> np.uint64(29))) + srt[:, k] * _HASH_MUL[k]
    order = np.argsort(h, kind="stable")                       # stable: first proposer first
    hs = h[order]
    ss = srt[order]
    if np.any((hs[1:] == hs[:-1]) & np.any(ss[1:] != ss[:-1], axis=1)):
        # two different quads share a hash: sort by the node tuples themselves
        order = np.lexsort((srt[:, 3], srt[:, 2], srt[:, 1], srt[:, 0]))
        ss = srt[order]
        hs = np.zeros(len(order), dtype=np.uint64)
    new_group = np.ones(len(order), dtype=bool)
    new_group[1:] = (hs[1:] != hs[:-1]) | np.any(ss[1:] != ss[:-1], axis=1)
    gid = np.cumsum(new_group) - 1
    nface = int(gid[-1]) + 1
    counts = np.bincount(gid, minlength=nface)
    if counts.max() > 2:
        raise ValueError("non-manifold mesh: a quad is shared by more than two cells")
    first = order[new_group]                                   # candidate index of the first proposer
    # faces numbered in order of their first proposer (cell order, then slot order)
    face_rank = np.argsort(first, kind="stable")
    first_sorted = first[face_rank]
    gid_to_face = np.empty(nface, dtype=np.int64)
    gid_to_face[face_rank] = np.arange(nface)
    cand_face = np.empty(len(order), dtype=np.int64)
    cand_face[order] = gid_to_face[gid]
    face_nodes = cand[first_sorted]
    face_cells = np.full((nface, 2), -1, dtype=np.int64)
    cand_cell = np.repeat(np.arange(ncell), 6)
    face_cells[:, 0] = cand_cell[first_sorted]
    is_first = np.zeros(len(order), dtype=bool)
    is_first[first_sorted] = True
    second = np.nonzero(~is_first)[0]
    face_cells[cand_face[second], 1] = cand_cell[second]
    cell_faces = cand_face.reshape(ncell, 6)
    return face_nodes.astype(np.int32), face_cells.astype(np.int32), cell_faces.astype(np.int32)


def _finish(node_xyz, cell_nodes, face_nodes, face_cells, cell_faces):
    nface = face_nodes.shape[0]
    ncell = cell_nodes.shape[0]
    return dict(
        node_xyz=np.ascontiguousarray(node_xyz, dtype=np.float64),
        cell_nodes=np.ascontiguousarray(cell_nodes, dtype=np.int32),
        cell_faces=np.ascontiguousarray(cell_faces, dtype=np.int32),
        cell_type=np.zeros(ncell, dtype=np.int8),
        cell_tvd=np.ones(ncell, dtype=np.uint8),
        face_nodes=np.ascontiguousarray(face_nodes, dtype=np.int32),
        face_cells=np.ascontiguousarray(face_cells, dtype=np.int32),
        face_type=np.zeros(nface, dtype=np.int8),
        face_surf=np.zeros(nface, dtype=np.int8),
        face_bc=np.full(nface, -1, dtype=np.int32),
        bc_vals=np.zeros((0, 10), dtype=np.float64),
        node_amp=None,
        node_phase=None,
    )


def cube_mesh(n: int, length: float = 1.0) -> dict:
    """Unit cube of n^3 hexahedra on [0, length]^3; every boundary face Outer_Soft."""
    return box_mesh(n, n, n, (length, length, length))


def box_mesh(nx: int, ny: int, nz: int, lengths=(1.0, 1.0, 1.0)) -> dict:
    """Box of nx x ny x nz hexahedra on [0, lx] x [0, ly] x [0, lz]; every
    boundary face Outer_Soft."""
    gx = np.arange(nx + 1, dtype=np.float64) * (lengths[0] / nx)
    gy = np.arange(ny + 1, dtype=np.float64) * (lengths[1] / ny)
    gz = np.arange(nz + 1, dtype=np.float64) * (lengths[2] / nz)
    X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
    node_xyz = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)

    def nid(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k

    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    cell_nodes = np.stack([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
                           nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)],
                          axis=1)
    fn, fc, cf = build_faces(cell_nodes)
    mesh = _finish(node_xyz, cell_nodes, fn, fc, cf)
    mesh["face_type"][fc[:, 1] < 0] = 3  # Outer_Soft
    return mesh


def cubed_sphere_directions(nq: int):
    """Unit directions of the (6 nq^2 + 2) nodes and the 6 nq^2 quads of an equiangular cubed sphere.

    Quads are listed counter-clockwise seen from outside."""
    L = nq
    # lattice points on the surface of the cube [0, L]^3
    idx = np.arange(L + 1)
    I, J, K = np.meshgrid(idx, idx, idx, indexing="ij")
    on = (I == 0) | (I == L) | (J == 0) | (J == L) | (K == 0) | (K == L)
    pts = np.stack([I[on], J[on], K[on]], axis=1)
    lut = -np.ones((L + 1,) * 3, dtype=np.int64)
    lut[pts[:, 0], pts[:, 1], pts[:, 2]] = np.arange(len(pts))
    t = np.tan(np.pi / 4 * (2.0 * pts / L - 1.0))
    # on the face where a coordinate is at 0 or L, that coordinate maps to -1/+1 exactly
    t = np.where(pts == 0, -1.0, np.where(pts == L, 1.0, t))
    dirs = t / np.linalg.norm(t, axis=1, keepdims=True)
    quads = []
    a = np.arange(L)
    A, B = np.meshgrid(a, a, indexing="ij")
    A, B = A.ravel(), B.ravel()
    for axis in range(3):
        for side in (0, L):
            u, v = [d for d in range(3) if d != axis]
            def q(da, db):
                c = np.zeros((len(A), 3), dtype=np.int64)
                c[:, axis] = side
                c[:, u] = A + da
                c[:, v] = B + db
                return lut[c[:, 0], c[:, 1], c[:, 2]]
            quad = np.stack([q(0, 0), q(1, 0), q(1, 1), q(0, 1)], axis=1)
            # orient counter-clockwise seen from outside: (e_u x e_v) . outward
            sign = np.cross(np.eye(3)[u], np.eye(3)[v])[axis] * (1 if side == L else -1)
            if sign < 0:
                quad = quad[:, ::-1]
            quads.append(quad)
    return dirs, np.concatenate(quads, axis=0)


def shell_mesh(nq: int, nlayer: int, r0: float = 1.0, r1: float = 100.0, outer_hard_x: float = 0.0,
               radii: np.ndarray | None = None) -> dict:
    """Spherical shell of 6 nq^2 x nlayer hexahedra with geometric radial spacing
    (or the nlayer + 1 node radii `radii`, from the inner sphere outwards).

    Inner sphere faces are Inner_Hard, outer faces Outer_Hard where the face
    centre has x > outer_hard_x (the inflow side) and Outer_Soft elsewhere —
    the typing rule of Setka::Init_boundary_grans (Setka_physics.cpp:208-236).
    Returns the mesh plus `node_layer` and `node_ray` (per-node indices)."""
    dirs, quads = cubed_sphere_directions(nq)
    ns = dirs.shape[0]
    if radii is None:
        radii = r0 * (r1 / r0) ** (np.arange(nlayer + 1) / nlayer)
    radii = np.asarray(radii, dtype=np.float64)
    assert radii.shape == (nlayer + 1,) and np.all(np.diff(radii) > 0)
    r0 = radii[0]
    node_xyz = (radii[:, None, None] * dirs[None, :, :]).reshape(-1, 3)
    nq_ = quads.shape[0]
    lay = np.arange(nlayer)
    base = (lay[:, None, None] * ns + quads[None, :, :]).reshape(-1, 4)
    cell_nodes = np.concatenate([base, base + ns], axis=1)
    fn, fc, cf = build_faces(cell_nodes)
    mesh = _finish(node_xyz, cell_nodes, fn, fc, cf)
    bnd = fc[:, 1] < 0
    cent = node_xyz[fn].mean(axis=1)
    rr = np.linalg.norm(cent, axis=1)
    inner = bnd & (rr < np.sqrt(r0 * radii[1]))
    outer = bnd & ~inner
    mesh["face_type"][inner] = 1
    mesh["face_type"][outer & (cent[:, 0] > outer_hard_x)] = 2
    mesh["face_type"][outer & ~(cent[:, 0] > outer_hard_x)] = 3
    mesh["node_layer"] = np.repeat(np.arange(nlayer + 1), ns)
    mesh["node_ray"] = np.tile(np.arange(ns), nlayer + 1)
    mesh["cell_layer"] = np.repeat(lay, nq_)
    mesh["radii"] = radii
    return mesh


def a_luch_radii(law: dict, R2: float, R3: float, R4: float) -> np.ndarray:
    """Node radii along a ray under the A_Luch law of Luch::dvigenie
    (TITAN/source/Luch.cpp:9-152) with the TS, HP and BS at R2, R3, R4: the
    M0 + M1 + M2 + M3 + M4 + 5 radii from R0 to R5 (Geo_param's M0..M4, R0,
    R1, R5, da1..da5 in `law`), for building a mesh the law leaves in place."""
    M0, M1, M11, M2, M3, M4 = (int(law[k]) for k in ("M0", "M1", "M11", "M2", "M3", "M4"))
    R0, R1, R5 = law["R0"], law["R1"], law["R5"]
    out = [R0 + j * (R1 - R0) / M0 for j in range(M0)] + [R1]
    out += [R1 + (j + 1) * (R2 - R1) / (M1 + 1) for j in range(M1)] + [R2]
    dr = (R2 - R1) / (M1 + 1)
    out += [R2 + dr * (j + 1) for j in range(M11)]
    a, b = law["da1"], law["da2"]
    for j in range(M2 - M11):
        s = (j + 1.0) / (M2 - M11 + 1.0)
        ss = s * (a * (1.0 - 3.0 * s + 2.0 * s * s) ** 2 +
                  s * (7.0 + b * (1.0 - 2.0 * s) ** 2 * (-1.0 + s) - 2.0 * s * (9.0 + 2.0 * s * (-5.0 + 2.0 * s))))
        out.append(R2 + dr * M11 + (R3 - R2 - dr * M11) * ss)
    out.append(R3)
    a, b = law["da3"], law["da4"]
    for j in range(M3):
        s = (j + 1.0) / (M3 + 1.0)
        out.append(R3 + (R4 - R3) * s * (a - (2.0 * a + b - 3.0) * s + (a + b - 2.0) * s * s))
    out.append(R4)
    a, b = law["da5"], 2.0
    for j in range(M4):
        s = (j + 1.0) / (M4 + 1.0)
        out.append(R4 + (R5 - R4) * (a * s - (3.0 * a + b - 4.0) * s ** 3 + (2.0 * a + b - 3.0) * s ** 4))
    out.append(R5)
    return np.array(out)


def shell_rays(mesh: dict) -> np.ndarray:
    """The shell's rays (Luch): node ids [6 nq^2 + 2, nlayer + 1], each a radial
    line of nodes from the inner sphere outwards."""
    layer, ray = mesh["node_layer"], mesh["node_ray"]
    out = np.empty((int(ray.max()) + 1, int(layer.max()) + 1), dtype=np.int32)
    out[ray, layer] = np.arange(len(ray), dtype=np.int32)
    return out


def mark_shell_surface(mesh: dict, layer: int, kind: int) -> None:
    """face_surf = kind (1 TS, 2 HP, 3 BS, Type_Gran_surf) on the spherical
    faces whose nodes all lie on node layer `layer` (an interior layer)."""
    on = np.all(mesh["node_layer"][mesh["face_nodes"]] == layer, axis=1)
    assert on.any() and not (mesh["face_type"][on] != 0).any(), "an interior node layer"
    mesh["face_surf"][on] = kind


def hex_geometry(mesh: dict, xyz: np.ndarray | None = None):
    """numpy geometry (cell centres, volumes, face centres, normals, areas) for tests."""
    xyz = mesh["node_xyz"] if xyz is None else xyz
    cn, fnd, fcl = mesh["cell_nodes"], mesh["face_nodes"], mesh["face_cells"]
    cc = xyz[cn].mean(axis=1)
    P = xyz[fnd]
    fc = P.mean(axis=1)
    area = 0.5 * np.linalg.norm(np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0]), axis=1) + \
        0.5 * np.linalg.norm(np.cross(P[:, 3] - P[:, 0], P[:, 2] - P[:, 0]), axis=1)
    m1, m2, m3 = (P[:, 0] + P[:, 1]) / 2, (P[:, 1] + P[:, 2]) / 2, (P[:, 2] + P[:, 3]) / 2
    nrm = np.cross(m2 - m1, m3 - m1)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    flip = np.sum(nrm * (cc[fcl[:, 0]] - fc), axis=1) > 0
    nrm[flip] *= -1
    return cc, fc, nrm, area
