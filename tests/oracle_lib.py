"""ctypes bindings for the oracle (test infrastructure only).

* ``oracle/liboracle.so``         — the CPU restatement of the plasma step
  (oracle/titan_oracle.cpp), built by ``make -C oracle``.
* ``oracle/_ref/libtitan_ref.so`` — the reference's own Riemann solver
  (TITAN/source/Phys_param.cpp compiled unmodified), built by
  ``make -C oracle ref`` where the reference tree is present.

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module; the shipped library never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")
REF_SO = os.path.join(ORACLE_DIR, "_ref", "libtitan_ref.so")
REF_RUN = os.path.join(ORACLE_DIR, "_ref", "run")

D = ctypes.POINTER(ctypes.c_double)
I32 = ctypes.POINTER(ctypes.c_int32)
I8 = ctypes.POINTER(ctypes.c_int8)
U8 = ctypes.POINTER(ctypes.c_uint8)

NV = 10


def _p(a, t=D):
    return None if a is None else a.ctypes.data_as(t)


class OMesh(ctypes.Structure):
    _fields_ = [
        ("nnode", ctypes.c_int64), ("ncell", ctypes.c_int64), ("nface", ctypes.c_int64),
        ("cell_nodes", I32), ("cell_faces", I32), ("cell_type", I8), ("cell_tvd", U8),
        ("face_nodes", I32), ("face_cells", I32), ("face_type", I8), ("face_surf", I8),
        ("face_method", I8), ("face_bc", I32), ("bc_vals", D), ("node_amp", D), ("node_phase", D),
        ("face_tvd", I32),
        ("ray_nodes", I32), ("ray_r0", D), ("ray_dir", D), ("nray", ctypes.c_int64), ("ray_len", ctypes.c_int64),
        ("face_nodt", I8), ("surf_centre", D), ("ray_law", D),
    ]

# The fields of titan_ray_law (the A_Luch law), in the oracle's order.
RAY_LAW_KEYS = ("M0", "M1", "M11", "M2", "M3", "M4", "R0", "R1", "R5", "da1", "da2", "da3", "da4", "da5")


class OParams(ctypes.Structure):
    _fields_ = [
        ("gamma", ctypes.c_double), ("KFL", ctypes.c_double), ("velosity_inf", ctypes.c_double),
        ("omega", ctypes.c_double), ("par_a_2", ctypes.c_double), ("par_n_H_LISM", ctypes.c_double),
        ("par_Kn", ctypes.c_double), ("beta_switch", ctypes.c_double),
        ("move", ctypes.c_int32), ("soft_fixups", ctypes.c_int32), ("method_policy", ctypes.c_int32),
        ("npassive", ctypes.c_int32), ("nh", ctypes.c_int32), ("TS_hard", ctypes.c_int32),
        ("contact_hard", ctypes.c_int32), ("tvd", ctypes.c_int32), ("snos_on_hp", ctypes.c_int32),
        ("bn_in_p_on_hp", ctypes.c_int32), ("surface_motion", ctypes.c_int32),
        ("move_TS", ctypes.c_int32), ("move_HP", ctypes.c_int32), ("move_BS", ctypes.c_int32),
        ("null_bn_on_HP", ctypes.c_int32), ("pad2", ctypes.c_int32),
        ("velocity_TS", ctypes.c_double), ("velocity_HP", ctypes.c_double), ("velocity_BS", ctypes.c_double),
        ("sglag_TS", ctypes.c_int32), ("sglag_HP", ctypes.c_int32), ("sglag_BS", ctypes.c_int32),
        ("hp_tail", ctypes.c_int32), ("sglag_TS_k_sphere", ctypes.c_double), ("sglag_HP_k_sphere", ctypes.c_double),
        ("sglag_BS_k", ctypes.c_double),
    ]

# The surface-tracking fields of OParams (titan_surface_params on the library side).
SURFACE_KEYS = ("move_TS", "move_HP", "move_BS", "null_bn_on_HP", "velocity_TS", "velocity_HP", "velocity_BS",
                "sglag_TS", "sglag_HP", "sglag_BS", "sglag_TS_k_sphere", "sglag_HP_k_sphere", "sglag_BS_k", "hp_tail")


class OStepInfo(ctypes.Structure):
    _fields_ = [("steps_done", ctypes.c_int64), ("err_code", ctypes.c_int64), ("err_index", ctypes.c_int64),
                ("n_rho_floor", ctypes.c_int64), ("n_p_floor", ctypes.c_int64)]


_oracle = None
_ref = None


def build_oracle(ref: bool = False) -> None:
    """Build the oracle (and, when asked and the reference tree exists, the reference solver)."""
    subprocess.run(["make", "-s", "-C", ORACLE_DIR, "all"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", ORACLE_DIR, "ref"], check=True)


def oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        lib = ctypes.CDLL(ORACLE_SO)
        lib.oracle_chlld.argtypes = [ctypes.c_int, D, ctypes.c_double, D, D, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, D, D, D, D, D, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        lib.oracle_chlld.restype = ctypes.c_int
        lib.oracle_chlld_batch.argtypes = [ctypes.c_int64, I32, D, D, D, D, D, D, ctypes.c_double, I32]
        lib.oracle_geometry.argtypes = [ctypes.POINTER(OMesh), D, D, D, D, D, D]
        lib.oracle_go.argtypes = [ctypes.POINTER(OMesh), ctypes.POINTER(OParams), D, D, D, D,
                                  ctypes.c_int64, D, ctypes.POINTER(OStepInfo)]
        lib.oracle_go.restype = ctypes.c_int
        lib.oracle_face_fluxes.argtypes = [ctypes.POINTER(OMesh), ctypes.POINTER(OParams), D, D, D,
                                           ctypes.c_double, D, ctypes.POINTER(ctypes.c_int)]
        lib.oracle_face_fluxes.restype = ctypes.c_double
        lib.oracle_sources.argtypes = [ctypes.POINTER(OMesh), ctypes.POINTER(OParams), D, D, D]
        lib.oracle_move_nodes.argtypes = [ctypes.POINTER(OMesh), ctypes.POINTER(OParams), D, D,
                                          ctypes.c_double, ctypes.c_double]
        lib.oracle_num_threads.restype = ctypes.c_int
        lib.oracle_set_reference_riemann.argtypes = [ctypes.c_void_p]
        lib.oracle_tvd_neighbours.argtypes = [ctypes.POINTER(OMesh), D, I32]
        lib.oracle_ray_geometry.argtypes = [ctypes.POINTER(OMesh), D, D, D]
        lib.oracle_surface_centres.argtypes = [ctypes.POINTER(OMesh), D, D]
        lib.oracle_godunov.argtypes = [D, ctypes.c_double, D, D, ctypes.c_int, ctypes.c_double, D, D]
        lib.oracle_godunov.restype = ctypes.c_int
        lib.oracle_face_states.argtypes = [ctypes.POINTER(OMesh), ctypes.POINTER(OParams), D, D, D, I8]
        _oracle = lib
    return _oracle


def use_reference_riemann(gamma: float | None) -> bool:
    """Installs the reference's own compiled Phys_param::chlld as the oracle
    step's Riemann solver (gamma: the step's adiabatic index), or removes it
    (None). Returns whether the reference solver is in use."""
    lib = oracle()
    if gamma is None or not ref_available():
        lib.oracle_set_reference_riemann(None)
        return False
    try:
        r = ref()
    except (OSError, RuntimeError):  # a reference build that does not load here
        lib.oracle_set_reference_riemann(None)
        return False
    r.titan_ref_set_gamma(float(gamma))
    lib.oracle_set_reference_riemann(ctypes.cast(r.titan_ref_chlld, ctypes.c_void_p).value)
    return True


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    """The reference's compiled Phys_param (raises if it was not built)."""
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(REF_SO)
        lib.titan_ref_init.argtypes = [ctypes.c_char_p]
        lib.titan_ref_init.restype = ctypes.c_int
        rc = lib.titan_ref_init(REF_RUN.encode())
        if rc != 0:
            raise RuntimeError(f"titan_ref_init failed: {rc}")
        lib.titan_ref_chlld.argtypes = [ctypes.c_int, D, ctypes.c_double, D, D, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, D, D, D, D, D, ctypes.c_int, ctypes.c_int]
        lib.titan_ref_set_gamma.argtypes = [ctypes.c_double]
        lib.titan_ref_godunov.argtypes = [D, ctypes.c_double, D, D, ctypes.c_int, D, D]
        lib.titan_ref_plasma_components_1.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                      ctypes.c_double, D]
        _ref = lib
    return _ref


def godunov(lib_kind: str, nrm, w, q1, q2, contact=0, gamma=5.0 / 3.0):
    """One exact Godunov solve (Phys_param::Godunov_Solver_Alexashov) through the
    oracle ('oracle') or the reference ('ref'): (flux[5], ds[3] = dsl, dsc, dsr, rc)."""
    nrm = np.ascontiguousarray(nrm, dtype=np.float64)
    qa = np.zeros(8)
    qb = np.zeros(8)
    qa[:len(q1)] = q1
    qb[:len(q2)] = q2
    out, ds = np.zeros(5), np.zeros(3)
    if lib_kind == "ref":
        r = ref()
        r.titan_ref_set_gamma(gamma)
        r.titan_ref_godunov(_p(nrm), float(w), _p(qa), _p(qb), int(contact), _p(out), _p(ds))
        rc = 0
    else:
        rc = oracle().oracle_godunov(_p(nrm), float(w), _p(qa), _p(qb), int(contact), float(gamma), _p(out), _p(ds))
    return out, ds, rc


def random_godunov_cases(n: int, seed: int = 0):
    """Face problems spread over the exact solver's four wave patterns (two
    shocks, shock + rarefaction, two rarefactions, vacuum), both pressure
    orders, moving faces: (nrm [n,3], w [n], q1 [n,5], q2 [n,5])."""
    rng = np.random.default_rng(seed)
    nrm = rng.standard_normal((n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    w = 0.2 * rng.standard_normal(n)
    q1, q2 = np.zeros((n, 5)), np.zeros((n, 5))
    for q in (q1, q2):
        q[:, 0] = np.exp(rng.uniform(-3, 1, n))
        q[:, 4] = np.exp(rng.uniform(-4, 1, n))
        q[:, 1:4] = 0.5 * rng.standard_normal((n, 3))
    # relative normal velocity from strongly colliding to strongly separating
    du = rng.uniform(-12.0, 6.0, n)
    q1[:, 1:4] += (0.5 * du)[:, None] * nrm
    q2[:, 1:4] -= (0.5 * du)[:, None] * nrm
    return nrm, w, q1, q2


def chlld(lib_kind: str, n_state, nrm, w, q1, q2, *, null_bn=0, n_disc=0, kl=(), kr=(), left_ydar=0,
          contact=0, gamma=5.0 / 3.0):
    """One Riemann-solver call through the oracle ('oracle') or the reference ('ref').

    Returns (flux[8], konvect[nk], ds[3] = (dsl, dsc, dsr), rc)."""
    nrm = np.ascontiguousarray(nrm, dtype=np.float64)
    q1 = np.ascontiguousarray(q1, dtype=np.float64)
    q2 = np.ascontiguousarray(q2, dtype=np.float64)
    nk = len(kl)
    kla = np.ascontiguousarray(kl if nk else [0.0], dtype=np.float64)
    kra = np.ascontiguousarray(kr if nk else [0.0], dtype=np.float64)
    out = np.zeros(8)
    kout = np.zeros(max(nk, 1))
    ds = np.zeros(3)
    if lib_kind == "ref":
        r = ref()
        r.titan_ref_set_gamma(gamma)
        r.titan_ref_chlld(int(n_state), _p(nrm), float(w), _p(q1), _p(q2), int(null_bn), int(n_disc), nk,
                          _p(kla), _p(kra), _p(out), _p(kout), _p(ds), int(left_ydar), int(contact))
        rc = 0
    else:
        rc = oracle().oracle_chlld(int(n_state), _p(nrm), float(w), _p(q1), _p(q2), int(null_bn), int(n_disc),
                                   nk, _p(kla), _p(kra), _p(out), _p(kout), _p(ds), int(left_ydar),
                                   int(contact), float(gamma))
    return out, kout[:nk], ds, rc


def random_riemann_cases(n: int, seed: int, *, weak_bn_frac=0.15, x_normal_frac=0.15):
    """Seeded random face problems covering every HLLD zone and both get_bazis branches."""
    rng = np.random.default_rng(seed)
    q1 = np.empty((n, 8))
    q2 = np.empty((n, 8))
    for q in (q1, q2):
        q[:, 0] = np.exp(rng.normal(0.0, 1.0, n))
        q[:, 1:4] = rng.normal(0.0, 1.0, (n, 3))
        q[:, 4] = np.exp(rng.normal(0.0, 1.0, n))
        q[:, 5:8] = rng.normal(0.0, 2.0, (n, 3))
    nrm = rng.normal(size=(n, 3))
    k = int(n * x_normal_frac)
    nrm[:k] = np.array([1.0, 0.0, 0.0]) + 0.05 * rng.normal(size=(k, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    # make some faces carry (almost) no normal field: |B_n| below epsb
    kb = int(n * weak_bn_frac)
    for q in (q1, q2):
        bn = np.sum(q[k:k + kb, 5:8] * nrm[k:k + kb], axis=1, keepdims=True)
        q[k:k + kb, 5:8] -= bn * nrm[k:k + kb]
    w = rng.normal(0.0, 1.5, n)
    w[rng.random(n) < 0.3] = 0.0
    return nrm, w, q1, q2


class OracleRun:
    """The oracle's step loop (oracle_go) on a mesh dict of titan_c-_b200.mesh."""

    def __init__(self, mesh: dict, params: dict, surface: dict | None = None, rays: np.ndarray | None = None,
                 ray_law: dict | None = None):
        """surface / rays: surface-tracking node motion (the SURFACE_KEYS of
        `surface`, rays [nray, ray_len] node ids from the inner end) instead of
        the prescribed radial law; ray_law: the A_Luch law (RAY_LAW_KEYS) for
        the rays instead of the fraction rule."""
        self._keep = {}

        def keep(name, a, dt):
            arr = None if a is None else np.ascontiguousarray(a, dtype=dt)
            self._keep[name] = arr
            return arr

        self.xyz = np.ascontiguousarray(mesh["node_xyz"], dtype=np.float64).copy()
        m = OMesh()
        m.nnode, m.ncell, m.nface = self.xyz.shape[0], mesh["cell_nodes"].shape[0], mesh["face_nodes"].shape[0]
        m.cell_nodes = _p(keep("cn", mesh["cell_nodes"], np.int32), I32)
        m.cell_faces = _p(keep("cf", mesh["cell_faces"], np.int32), I32)
        m.cell_type = _p(keep("ct", mesh["cell_type"], np.int8), I8)
        m.cell_tvd = _p(keep("cv", mesh["cell_tvd"], np.uint8), U8)
        m.face_nodes = _p(keep("fn", mesh["face_nodes"], np.int32), I32)
        m.face_cells = _p(keep("fc", mesh["face_cells"], np.int32), I32)
        m.face_type = _p(keep("ft", mesh["face_type"], np.int8), I8)
        m.face_surf = _p(keep("fs", mesh["face_surf"], np.int8), I8)
        self.face_method = keep("fm", np.full(m.nface, 0, dtype=np.int8), np.int8)
        self.face_method[:] = np.where(mesh["face_surf"] != 0, 3, 0)   # Gran::Get_method
        m.face_method = _p(self.face_method, I8)
        m.face_bc = _p(keep("fb", mesh["face_bc"], np.int32), I32)
        bc = keep("bc", mesh["bc_vals"], np.float64)
        m.bc_vals = _p(bc) if bc.shape[0] else None
        m.node_amp = _p(keep("amp", mesh.get("node_amp"), np.float64))
        m.node_phase = _p(keep("ph", mesh.get("node_phase"), np.float64))
        self.mesh = m
        p = OParams()
        for k, _ in OParams._fields_:
            if k not in ("pad2", "surface_motion") + SURFACE_KEYS:
                setattr(p, k, params[k])
        if surface is not None:
            p.surface_motion = 1
            for k in SURFACE_KEYS:
                setattr(p, k, surface.get(k, 0))
            rn = keep("rays", rays, np.int32)
            m.ray_nodes = _p(rn, I32)
            m.nray, m.ray_len = rn.shape
            r0 = keep("ray_r0", np.empty(rn.shape), np.float64)
            rd = keep("ray_dir", np.empty((rn.shape[0], 3)), np.float64)
            oracle().oracle_ray_geometry(ctypes.byref(m), _p(self.xyz), _p(r0), _p(rd))
            m.ray_r0, m.ray_dir = _p(r0), _p(rd)
            if ray_law is not None:
                m.ray_law = _p(keep("ray_law", [float(ray_law[k]) for k in RAY_LAW_KEYS], np.float64))
            if p.sglag_TS or p.sglag_HP:
                sc = keep("surf_centre", np.zeros((m.nnode, 3)), np.float64)
                oracle().oracle_surface_centres(ctypes.byref(m), _p(self.xyz), _p(sc))
                m.surf_centre = _p(sc)
        self.params = p
        self.face_tvd = None
        if p.tvd:
            self.face_tvd = keep("tvd", np.empty((m.nface, 2), dtype=np.int32), np.int32)
            oracle().oracle_tvd_neighbours(ctypes.byref(m), _p(self.xyz), _p(self.face_tvd, I32))
            m.face_tvd = _p(self.face_tvd, I32)
        self.ncell = m.ncell
        self.clock = np.array([1e-5, 0.0])
        self.hf = None
        self.src = None

    def set_face_method(self, ns):
        self.face_method[:] = np.asarray(ns, dtype=np.int8)

    def set_cfl_faces(self, exclude):
        """Faces (1) left out of the CFL minimum; None: every interior face counts."""
        a = None if exclude is None else np.ascontiguousarray(exclude, dtype=np.int8)
        self._keep["nodt"] = a
        self.mesh.face_nodt = _p(a, I8)

    def go(self, state: np.ndarray, steps: int) -> OStepInfo:
        """Advances `state` ([10, C], modified in place) by `steps` steps."""
        assert state.flags.c_contiguous and state.dtype == np.float64
        info = OStepInfo()
        oracle().oracle_go(ctypes.byref(self.mesh), ctypes.byref(self.params), _p(state), _p(self.xyz),
                           _p(self.hf), _p(self.src), int(steps), _p(self.clock), ctypes.byref(info))
        return info

    def geometry(self, xyz=None):
        xyz = self.xyz if xyz is None else np.ascontiguousarray(xyz)
        nc, nf = self.mesh.ncell, self.mesh.nface
        cc, vol = np.empty((nc, 3)), np.empty(nc)
        fc, fn, fa = np.empty((nf, 3)), np.empty((nf, 3)), np.empty(nf)
        oracle().oracle_geometry(ctypes.byref(self.mesh), _p(xyz), _p(cc), _p(vol), _p(fc), _p(fn), _p(fa))
        return dict(cell_center=cc, cell_volume=vol, face_center=fc, face_normal=fn, face_area=fa)

    def face_states(self, state: np.ndarray):
        """(LR [nface, 2, 10] reconstructed face states of interior faces, used [nface] second order)."""
        nf = self.mesh.nface
        LR = np.zeros((nf, 2, NV))
        used = np.zeros(nf, dtype=np.int8)
        oracle().oracle_face_states(ctypes.byref(self.mesh), ctypes.byref(self.params),
                                    _p(np.ascontiguousarray(state)), _p(self.xyz), _p(LR), _p(used, I8))
        return LR, used

    def face_fluxes(self, state: np.ndarray, time: float = 1e-5):
        """Face fluxes (11 per face) of `state` at the current nodes (stationary w)."""
        fl = np.empty((self.mesh.nface, 11))
        err = ctypes.c_int(0)
        dtn = oracle().oracle_face_fluxes(ctypes.byref(self.mesh), ctypes.byref(self.params), _p(state),
                                          _p(self.xyz), _p(self.xyz), float(time), _p(fl), ctypes.byref(err))
        return fl, dtn, err.value


def renumbered_mesh(mesh: dict, cell_n2o, face_n2o, node_n2o) -> dict:
    """The mesh in a context's renumbering (new index -> original index arrays,
    PlasmaStep.permutation()): every object moved to its new index and every
    reference rewritten, the per-face node order and per-cell face order kept."""
    c_o2n = np.empty_like(cell_n2o)
    c_o2n[cell_n2o] = np.arange(len(cell_n2o), dtype=cell_n2o.dtype)
    f_o2n = np.empty_like(face_n2o)
    f_o2n[face_n2o] = np.arange(len(face_n2o), dtype=face_n2o.dtype)
    n_o2n = np.empty_like(node_n2o)
    n_o2n[node_n2o] = np.arange(len(node_n2o), dtype=node_n2o.dtype)
    fcl = mesh["face_cells"][face_n2o]
    fcl = np.where(fcl >= 0, c_o2n[np.maximum(fcl, 0)], -1).astype(np.int32)
    out = dict(
        node_xyz=np.ascontiguousarray(mesh["node_xyz"][node_n2o]),
        cell_nodes=n_o2n[mesh["cell_nodes"][cell_n2o]].astype(np.int32),
        cell_faces=f_o2n[mesh["cell_faces"][cell_n2o]].astype(np.int32),
        cell_type=mesh["cell_type"][cell_n2o], cell_tvd=mesh["cell_tvd"][cell_n2o],
        face_nodes=n_o2n[mesh["face_nodes"][face_n2o]].astype(np.int32), face_cells=fcl,
        face_type=mesh["face_type"][face_n2o], face_surf=mesh["face_surf"][face_n2o],
        face_bc=mesh["face_bc"][face_n2o], bc_vals=mesh["bc_vals"], node_amp=None, node_phase=None)
    return out, c_o2n


class OMcFaceDist(ctypes.Structure):
    _fields_ = [("nface", ctypes.c_int64), ("face", I32), ("side", I8), ("frame", D),
                ("leaf_ptr", ctypes.POINTER(ctypes.c_int64)), ("leaf_box", D), ("leaf_f", D)]


class OMcFaceTally(ctypes.Structure):
    _fields_ = [("nface", ctypes.c_int64), ("face", I32), ("side", I8), ("frame", D),
                ("leaf_ptr", ctypes.POINTER(ctypes.c_int64)), ("leaf_box", D), ("leaf_f", D), ("moments", D),
                ("unplaced", ctypes.POINTER(ctypes.c_int64))]


def mc_pass(mesh: dict, state: np.ndarray, params: dict, n_H: float, u_H, cp_H: float, n_particles: int,
            seed: int = 1, face_types: int = (1 << 2) | (1 << 3), max_cells: int = 1000000,
            face_dist: dict | None = None, face_tally: dict | None = None):
    """The oracle's Monte-Carlo pass on a stationary mesh: (tally [5, ncell],
    trace [n_particles, 8], inflow rate, lost). face_dist: tabulated inflow
    of some faces (face, side, frame, leaf_ptr, leaf_box, leaf_f; face ids in
    `mesh`'s numbering); face_tally: outgoing tallies (face, side, frame,
    leaf_ptr, leaf_box), whose results (leaf_f, moments, unplaced) are added
    to that dict."""
    run = OracleRun(mesh, params)
    st = np.ascontiguousarray(state, dtype=np.float64)
    C = run.mesh.ncell
    tally = np.empty((5, C))
    trace = np.empty((n_particles, 8))
    total = ctypes.c_double(0.0)
    lost = ctypes.c_int64(0)
    uH = np.ascontiguousarray(u_H, dtype=np.float64)
    L = oracle()
    L.oracle_mc_pass.restype = ctypes.c_int
    L.oracle_mc_pass.argtypes = [ctypes.POINTER(OMesh), D, D, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, D, ctypes.c_double, ctypes.c_uint32, ctypes.c_uint64,
                                 ctypes.c_int64, ctypes.c_int32, D, D, D, ctypes.POINTER(ctypes.c_int64),
                                 ctypes.POINTER(OMcFaceDist), ctypes.POINTER(OMcFaceTally)]
    fd, keep = None, []
    if face_dist is not None:
        arrs = dict(face=np.ascontiguousarray(face_dist["face"], dtype=np.int32),
                    side=np.ascontiguousarray(face_dist["side"], dtype=np.int8),
                    frame=np.ascontiguousarray(face_dist["frame"], dtype=np.float64),
                    leaf_ptr=np.ascontiguousarray(face_dist["leaf_ptr"], dtype=np.int64),
                    leaf_box=np.ascontiguousarray(face_dist["leaf_box"], dtype=np.float64),
                    leaf_f=np.ascontiguousarray(face_dist["leaf_f"], dtype=np.float64))
        keep.append(arrs)
        fd = OMcFaceDist(len(arrs["face"]), _p(arrs["face"], I32), _p(arrs["side"], I8), _p(arrs["frame"]),
                         arrs["leaf_ptr"].ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _p(arrs["leaf_box"]),
                         _p(arrs["leaf_f"]))
    ft = None
    if face_tally is not None:
        t = dict(face=np.ascontiguousarray(face_tally["face"], dtype=np.int32),
                 side=np.ascontiguousarray(face_tally["side"], dtype=np.int8),
                 frame=np.ascontiguousarray(face_tally["frame"], dtype=np.float64),
                 leaf_ptr=np.ascontiguousarray(face_tally["leaf_ptr"], dtype=np.int64),
                 leaf_box=np.ascontiguousarray(face_tally["leaf_box"], dtype=np.float64))
        nt = len(t["face"])
        t["leaf_f"] = np.zeros(int(t["leaf_ptr"][-1]))
        t["moments"] = np.zeros((nt, 3))
        t["unplaced"] = np.zeros(1, dtype=np.int64)
        keep.append(t)
        ft = OMcFaceTally(nt, _p(t["face"], I32), _p(t["side"], I8), _p(t["frame"]),
                          t["leaf_ptr"].ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _p(t["leaf_box"]),
                          _p(t["leaf_f"]), _p(t["moments"]),
                          t["unplaced"].ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    rc = L.oracle_mc_pass(ctypes.byref(run.mesh), _p(run.xyz), _p(st), int(params["npassive"]),
                          float(params["par_a_2"]), float(params["par_Kn"]), float(n_H), _p(uH), float(cp_H),
                          int(face_types), int(seed), int(n_particles), int(max_cells), _p(tally), _p(trace),
                          ctypes.byref(total), ctypes.byref(lost), ctypes.byref(fd) if fd is not None else None,
                          ctypes.byref(ft) if ft is not None else None)
    if rc:
        raise RuntimeError("oracle_mc_pass: no inflow faces")
    if ft is not None:
        face_tally.update(leaf_f=keep[-1]["leaf_f"], moments=keep[-1]["moments"],
                          unplaced=int(keep[-1]["unplaced"][0]))
    return tally, trace, total.value, lost.value
