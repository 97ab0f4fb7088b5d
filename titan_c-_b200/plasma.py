"""Python view of the C ABI, shaped like the reference's plasma loop.

``PlasmaStep`` owns one titan context: the flattened mesh (Setka's All_Cell /
All_Gran / All_Yzel), the cell state (Cell::parameters) and the step loop of
Setka::Go (TITAN/source/Setka_physics.cpp:1484-2278). ``chlld`` is the batched
form of Phys_param::chlld (TITAN/source/Phys_param.cpp:882-1878) on the GPU.
Errors surface as TitanError carrying the C status code.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import native as N


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class PlasmaStep:
    """One B200 context for a mesh; `go(steps)` advances the plasma."""

    def __init__(self, mesh: dict, params: dict):
        L = N.lib()
        self._keep = {}

        def keep(name, a, dt):
            arr = None if a is None else np.ascontiguousarray(a, dtype=dt)
            self._keep[name] = arr
            return arr

        xyz = keep("xyz", mesh["node_xyz"], np.float64)
        cn = keep("cn", mesh["cell_nodes"], np.int32)
        cf = keep("cf", mesh["cell_faces"], np.int32)
        ct = keep("ct", mesh["cell_type"], np.int8)
        cv = keep("cv", mesh["cell_tvd"], np.uint8)
        fnd = keep("fn", mesh["face_nodes"], np.int32)
        fcl = keep("fc", mesh["face_cells"], np.int32)
        ft = keep("ft", mesh["face_type"], np.int8)
        fs = keep("fs", mesh["face_surf"], np.int8)
        fb = keep("fb", mesh["face_bc"], np.int32)
        bc = keep("bc", mesh["bc_vals"], np.float64)
        amp = keep("amp", mesh.get("node_amp"), np.float64)
        ph = keep("ph", mesh.get("node_phase"), np.float64)
        self.ncell = cn.shape[0]
        self.nface = fnd.shape[0]
        self.nnode = xyz.shape[0]
        m = N.TitanMesh()
        m.nnode, m.ncell, m.nface, m.nbc = self.nnode, self.ncell, self.nface, bc.shape[0]
        m.node_xyz, m.cell_nodes, m.cell_faces = N.ptr(xyz), N.ptr(cn, N.I32), N.ptr(cf, N.I32)
        m.cell_type, m.cell_tvd = N.ptr(ct, N.I8), N.ptr(cv, N.U8)
        m.face_nodes, m.face_cells = N.ptr(fnd, N.I32), N.ptr(fcl, N.I32)
        m.face_type, m.face_surf, m.face_bc = N.ptr(ft, N.I8), N.ptr(fs, N.I8), N.ptr(fb, N.I32)
        m.bc_vals = N.ptr(bc) if bc.shape[0] else None
        m.node_amp, m.node_phase = N.ptr(amp), N.ptr(ph)
        p = N.TitanParams()
        for k, _ in N.TitanParams._fields_:
            setattr(p, k, params[k])
        self.params = dict(params)
        ctx = ctypes.c_void_p()
        N.check(L.titan_create(ctypes.byref(m), ctypes.byref(p), ctypes.byref(ctx)))
        self._ctx = ctx
        self._lib = L
        self._keep.clear()  # the library copied everything
        self.dt = 1e-5      # Setka::Go starts with time = 1e-5 (Setka_physics.cpp:1582)
        self.t = 0.0
        self.last_info = None

    # -- context management ------------------------------------------------
    def close(self):
        if getattr(self, "_ctx", None) is not None and self._ctx.value:
            self._lib.titan_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def ctx(self):
        return self._ctx

    # -- data --------------------------------------------------------------
    def set_face_method(self, n_state: np.ndarray):
        a = np.ascontiguousarray(n_state, dtype=np.int8)
        N.check(self._lib.titan_set_face_method(self._ctx, N.ptr(a, N.I8)))

    def set_surface_motion(self, rays: np.ndarray | None, **surface):
        """Surface-tracking node motion (titan_set_surface_motion): rays [nray,
        ray_len] node ids from the inner end; surface: velocity_TS/_HP/_BS,
        move_TS/_HP/_BS, null_bn_on_HP. rays None returns to the prescribed motion."""
        if rays is None:
            N.check(self._lib.titan_set_surface_motion(self._ctx, None, 0, 0, None))
            return
        sp = N.TitanSurfaceParams()
        for k, _ in N.TitanSurfaceParams._fields_:
            setattr(sp, k, surface.get(k, 0))
        r = np.ascontiguousarray(rays, dtype=np.int32)
        N.check(self._lib.titan_set_surface_motion(self._ctx, ctypes.byref(sp), r.shape[0], r.shape[1],
                                                   N.ptr(r, N.I32)))

    def set_ray_law(self, law: dict | None):
        """The A_Luch spacing law for the rays of set_surface_motion
        (titan_set_ray_law): M0, M1, M11, M2, M3, M4, R0, R1, R5, da1..da5;
        None returns to the fraction rule."""
        if law is None:
            N.check(self._lib.titan_set_ray_law(self._ctx, None))
            return
        g = N.TitanRayLaw()
        for k, _ in N.TitanRayLaw._fields_:
            if k != "pad":
                setattr(g, k, law[k])
        N.check(self._lib.titan_set_ray_law(self._ctx, ctypes.byref(g)))

    def set_halo(self, send_ids: np.ndarray, recv_ids: np.ndarray):
        """Cells this context sends to / receives from its peers in a sharded step (titan_set_halo)."""
        s = np.ascontiguousarray(send_ids, dtype=np.int32)
        r = np.ascontiguousarray(recv_ids, dtype=np.int32)
        N.check(self._lib.titan_set_halo(self._ctx, len(s), N.ptr(s, N.I32), len(r), N.ptr(r, N.I32)))

    def set_cfl_faces(self, exclude: np.ndarray | None):
        """Faces (1) whose CFL candidate is left out of dt (titan_set_cfl_faces); None: all count."""
        a = None if exclude is None else np.ascontiguousarray(exclude, dtype=np.int8)
        N.check(self._lib.titan_set_cfl_faces(self._ctx, N.ptr(a, N.I8)))

    def pack_halo(self, out_device_ptr: int):
        """The send cells' states, [n_send][8 + npassive], into a device buffer (address)."""
        N.check(self._lib.titan_pack_halo(self._ctx, ctypes.c_void_p(out_device_ptr)))

    def unpack_halo(self, in_device_ptr: int):
        """A device buffer [n_recv][8 + npassive] into the received cells."""
        N.check(self._lib.titan_unpack_halo(self._ctx, ctypes.c_void_p(in_device_ptr)))

    def upload_state(self, state: np.ndarray):
        a = np.ascontiguousarray(state, dtype=np.float64)
        assert a.shape == (N.NV, self.ncell)
        N.check(self._lib.titan_upload_state(self._ctx, N.ptr(a)))

    def download_state(self, out: np.ndarray | None = None) -> np.ndarray:
        # rows the context does not carry stay as given (zeros in a new array)
        out = np.zeros((N.NV, self.ncell)) if out is None else out
        N.check(self._lib.titan_download_state(self._ctx, N.ptr(out)))
        return out

    def upload_hfluids(self, h: np.ndarray):
        a = np.ascontiguousarray(h, dtype=np.float64)
        N.check(self._lib.titan_upload_hfluids(self._ctx, N.ptr(a)))

    def set_sources(self, s: np.ndarray | None):
        a = None if s is None else np.ascontiguousarray(s, dtype=np.float64)
        N.check(self._lib.titan_set_sources(self._ctx, N.ptr(a)))

    def go(self, steps: int) -> dict:
        """`steps` plasma steps; dt and t carry over between calls like Setka::Go's loop."""
        dt = ctypes.c_double(self.dt)
        t = ctypes.c_double(self.t)
        info = N.TitanStepInfo()
        rc = self._lib.titan_step(self._ctx, int(steps), ctypes.byref(dt), ctypes.byref(t), ctypes.byref(info))
        self.last_info = {k: getattr(info, k) for k, _ in N.TitanStepInfo._fields_}
        if rc == N.TITAN_OK:
            self.dt, self.t = dt.value, t.value
        N.check(rc)
        return self.last_info

    # -- the loop paced by the device (titan_set_clock / titan_step_async /
    # titan_dt_copy / titan_get_clock): ordered on self.stream(), no host wait
    def set_clock(self, dt: float | None = None, t: float | None = None):
        N.check(self._lib.titan_set_clock(self._ctx, float(self.dt if dt is None else dt),
                                          float(self.t if t is None else t)))

    def step_async(self, steps: int):
        N.check(self._lib.titan_step_async(self._ctx, int(steps)))

    def dt_copy(self, dev_ptr: int, into_clock: bool):
        """The device clock's dt to (False) or from (True) one double at dev_ptr."""
        N.check(self._lib.titan_dt_copy(self._ctx, ctypes.c_void_p(dev_ptr), int(into_clock)))

    def get_clock(self) -> dict:
        """Waits for the stream; dt and t of the device clock, and the run's info."""
        dt, t = ctypes.c_double(0.0), ctypes.c_double(0.0)
        info = N.TitanStepInfo()
        rc = self._lib.titan_get_clock(self._ctx, ctypes.byref(dt), ctypes.byref(t), ctypes.byref(info))
        self.last_info = {k: getattr(info, k) for k, _ in N.TitanStepInfo._fields_}
        if rc == N.TITAN_OK:
            self.dt, self.t = dt.value, t.value
        N.check(rc)
        return self.last_info

    def nodes(self) -> np.ndarray:
        out = np.empty((self.nnode, 3))
        N.check(self._lib.titan_download_nodes(self._ctx, N.ptr(out)))
        return out

    def geometry(self):
        cc = np.empty((self.ncell, 3))
        vol = np.empty(self.ncell)
        fc = np.empty((self.nface, 3))
        fn = np.empty((self.nface, 3))
        fa = np.empty(self.nface)
        N.check(self._lib.titan_download_geometry(self._ctx, N.ptr(cc), N.ptr(vol), N.ptr(fc), N.ptr(fn),
                                                  N.ptr(fa)))
        return dict(cell_center=cc, cell_volume=vol, face_center=fc, face_normal=fn, face_area=fa)

    def face_fluxes(self) -> np.ndarray:
        out = np.empty((self.nface, 11))
        N.check(self._lib.titan_download_face_fluxes(self._ctx, N.ptr(out)))
        return out

    def upload_nodes(self, xyz: np.ndarray):
        """Node coordinates [nnode, 3]; the geometry is formed again from them."""
        a = np.ascontiguousarray(xyz, dtype=np.float64)
        assert a.shape == (self.nnode, 3)
        N.check(self._lib.titan_upload_nodes(self._ctx, N.ptr(a)))

    def save_checkpoint(self, path: str, nodes: bool = True):
        """The state (and nodes) as a reference cell-parameter file (Setka::Save_cell_parameters)."""
        st = np.ascontiguousarray(self.download_state())
        xyz = np.ascontiguousarray(self.nodes()) if nodes else None
        N.check(self._lib.titan_write_cell_parameters(path.encode(), self.ncell, 8 + int(self.params["npassive"]), N.ptr(st),
                                                      self.nnode, N.ptr(xyz)))

    def load_checkpoint(self, path: str) -> dict:
        """A reference cell-parameter file (Setka::Download_cell_parameters): the
        plasma fields it holds replace the state; its node block, if any, the nodes."""
        st = np.ascontiguousarray(self.download_state())
        xyz = np.empty((self.nnode, 3))
        found = ctypes.c_int32(0)
        has_nodes = ctypes.c_int32(0)
        N.check(self._lib.titan_read_cell_parameters(path.encode(), self.ncell, self.nnode, N.ptr(st), N.ptr(xyz),
                                                     ctypes.byref(found), ctypes.byref(has_nodes)))
        self.upload_state(st)
        if has_nodes.value:
            self.upload_nodes(xyz)
        return {"fields": [n for k, n in enumerate(N.FIELDS) if found.value >> k & 1],
                "nodes": bool(has_nodes.value)}

    def tvd_neighbours(self) -> np.ndarray:
        """[nface, 2] second-order neighbours (AA, BB), original numbering, -1 when absent."""
        out = np.empty((self.nface, 2), dtype=np.int32)
        N.check(self._lib.titan_get_tvd_neighbours(self._ctx, N.ptr(out, N.I32)))
        return out

    def permutation(self):
        c = np.empty(self.ncell, dtype=np.int32)
        f = np.empty(self.nface, dtype=np.int32)
        n = np.empty(self.nnode, dtype=np.int32)
        N.check(self._lib.titan_get_permutation(self._ctx, N.ptr(c, N.I32), N.ptr(f, N.I32), N.ptr(n, N.I32)))
        return c, f, n

    @staticmethod
    def _mc_params(n_H, u_H, cp_H, n_particles, seed, face_types, max_cells):
        mp = N.TitanMcParams()
        mp.n_H, mp.cp_H = n_H, cp_H
        for k in range(3):
            mp.u_H[k] = u_H[k]
        mp.n_particles, mp.seed, mp.max_cells, mp.face_types = int(n_particles), int(seed), int(max_cells), face_types
        return mp

    def mc_sources(self, n_H: float, u_H, cp_H: float, n_particles: int, seed: int = 1,
                   face_types: int = (1 << 2) | (1 << 3), max_cells: int = 0, out: np.ndarray | None = None,
                   trace: np.ndarray | None = None):
        """Monte-Carlo neutrals through the current state: ([5, ncell] = n_H, S_m (3), S_E; info).
        `out`, a C-contiguous float64 [5, ncell] array, is filled in place when given;
        `trace`, a C-contiguous float64 [n_particles, 8] array, receives each neutral's end
        record (titan_mc_params.trace_out)."""
        mp = self._mc_params(n_H, u_H, cp_H, n_particles, seed, face_types, max_cells)
        if trace is not None:
            if trace.shape != (n_particles, 8) or trace.dtype != np.float64 or not trace.flags.c_contiguous:
                raise ValueError("trace must be a C-contiguous float64 array of shape (n_particles, 8)")
            mp.trace_out = trace.ctypes.data
        if out is None:
            out = np.empty((5, self.ncell))
        elif out.shape != (5, self.ncell) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of shape (5, ncell)")
        info = N.TitanMcInfo()
        N.check(self._lib.titan_mc_sources(self._ctx, ctypes.byref(mp), N.ptr(out), ctypes.byref(info)))
        return out, {k: getattr(info, k) for k, _ in N.TitanMcInfo._fields_}

    def set_mc_face_dist(self, face_dist: dict | None):
        """Tabulated velocity distributions of the neutrals entering through
        some faces (titan_set_mc_face_dist): face (original ids), side, frame
        [n, 9], leaf_ptr [n + 1], leaf_box [nleaf, 6], leaf_f [nleaf]; None
        removes them."""
        if face_dist is None:
            N.check(self._lib.titan_set_mc_face_dist(self._ctx, None))
            return
        arrs = dict(face=np.ascontiguousarray(face_dist["face"], dtype=np.int32),
                    side=np.ascontiguousarray(face_dist["side"], dtype=np.int8),
                    frame=np.ascontiguousarray(face_dist["frame"], dtype=np.float64),
                    leaf_ptr=np.ascontiguousarray(face_dist["leaf_ptr"], dtype=np.int64),
                    leaf_box=np.ascontiguousarray(face_dist["leaf_box"], dtype=np.float64),
                    leaf_f=np.ascontiguousarray(face_dist["leaf_f"], dtype=np.float64))
        d = N.TitanMcFaceDist(len(arrs["face"]), *(arrs[k].ctypes.data for k in
                                                   ("face", "side", "frame", "leaf_ptr", "leaf_box", "leaf_f")))
        N.check(self._lib.titan_set_mc_face_dist(self._ctx, ctypes.byref(d)))

    def set_mc_face_tally(self, face_tally: dict | None):
        """Outgoing distributions tallied on some faces (titan_set_mc_face_tally):
        face (original ids), side, frame [n, 9], leaf_ptr [n + 1], leaf_box
        [nleaf, 6]; None removes them."""
        if face_tally is None:
            N.check(self._lib.titan_set_mc_face_tally(self._ctx, None))
            self._ft_shape = None
            return
        arrs = dict(face=np.ascontiguousarray(face_tally["face"], dtype=np.int32),
                    side=np.ascontiguousarray(face_tally["side"], dtype=np.int8),
                    frame=np.ascontiguousarray(face_tally["frame"], dtype=np.float64),
                    leaf_ptr=np.ascontiguousarray(face_tally["leaf_ptr"], dtype=np.int64),
                    leaf_box=np.ascontiguousarray(face_tally["leaf_box"], dtype=np.float64))
        d = N.TitanMcFaceTally(len(arrs["face"]), *(arrs[k].ctypes.data for k in
                                                    ("face", "side", "frame", "leaf_ptr", "leaf_box")))
        N.check(self._lib.titan_set_mc_face_tally(self._ctx, ctypes.byref(d)))
        self._ft_shape = (len(arrs["face"]), int(arrs["leaf_ptr"][-1]))

    def mc_face_tally(self) -> dict:
        """The last pass's face tallies: leaf_f [nleaf], moments [n, 3] (n, Smu, nn), unplaced."""
        nt, nl = self._ft_shape
        f = np.empty(nl)
        mom = np.empty((nt, 3))
        u = ctypes.c_int64(0)
        N.check(self._lib.titan_get_mc_face_tally(self._ctx, N.ptr(f), N.ptr(mom), ctypes.byref(u)))
        return dict(leaf_f=f, moments=mom, unplaced=u.value)

    def mc_pass(self, n_H: float, u_H, cp_H: float, n_particles: int, seed: int = 1,
                face_types: int = (1 << 2) | (1 << 3), max_cells: int = 0) -> dict:
        """A Monte-Carlo pass whose sources stay on the device (for
        Closure.fallback_from_mc); returns the pass's info."""
        mp = self._mc_params(n_H, u_H, cp_H, n_particles, seed, face_types, max_cells)
        info = N.TitanMcInfo()
        N.check(self._lib.titan_mc_sources(self._ctx, ctypes.byref(mp), None, ctypes.byref(info)))
        return {k: getattr(info, k) for k, _ in N.TitanMcInfo._fields_}

    def autotune(self, reps: int = 5, cache: str | None = None) -> dict:
        """Times the launch-shape variants on this mesh and keeps the fastest."""
        N.check(self._lib.titan_autotune(self._ctx, int(reps), cache.encode() if cache else None))
        return self.tuning()

    def set_closure_overlap(self, on: bool):
        """Run the closure beside the face kernel (titan_set_closure_overlap)."""
        N.check(self._lib.titan_set_closure_overlap(self._ctx, int(bool(on))))

    def set_tuning(self, face_variant: int, cell_variant: int):
        N.check(self._lib.titan_set_tuning(self._ctx, int(face_variant), int(cell_variant)))

    def tuning(self) -> dict:
        v = [np.zeros(1, dtype=np.int32) for _ in range(5)]
        N.check(self._lib.titan_get_tuning(self._ctx, *[N.ptr(a, N.I32) for a in v]))
        keys = ["face_variant", "cell_variant", "face_block", "face_min_blocks", "cell_block"]
        return {k: int(a[0]) for k, a in zip(keys, v)}

    def stream(self) -> int:
        return int(self._lib.titan_stream(self._ctx) or 0)

    def set_profiling(self, on: bool):
        N.check(self._lib.titan_set_profiling(self._ctx, int(on)))

    def kernel_times(self) -> dict:
        cap = 16
        names = (ctypes.c_char_p * cap)()
        ms = np.zeros(cap)
        cnt = np.zeros(cap, dtype=np.int64)
        n = self._lib.titan_kernel_times(self._ctx, names, N.ptr(ms), N.ptr(cnt, N.I64), cap)
        return {names[i].decode(): (float(ms[i]), int(cnt[i])) for i in range(n)}

    def device_bytes(self) -> int:
        return int(self._lib.titan_device_bytes(self._ctx))


def chlld(n_state, nrm, w, q1, q2, *, flags: int = 0, precision: int = 64, gamma: float = 5.0 / 3.0):
    """Batched Phys_param::chlld on the GPU. Returns (flux [n,8], ds [n,3], rc [n])."""
    q1 = np.ascontiguousarray(q1, dtype=np.float64)
    q2 = np.ascontiguousarray(q2, dtype=np.float64)
    n = q1.shape[0]
    ns = np.ascontiguousarray(np.broadcast_to(np.asarray(n_state, dtype=np.int8), (n,)))
    nrm = np.ascontiguousarray(nrm, dtype=np.float64)
    w = np.ascontiguousarray(np.broadcast_to(np.asarray(w, dtype=np.float64), (n,)))
    flux = np.empty((n, 8))
    ds = np.empty((n, 3))
    rc = np.empty(n, dtype=np.int32)
    N.check(N.lib().titan_riemann_batch(n, N.ptr(ns, N.I8), N.ptr(nrm), N.ptr(w), N.ptr(q1), N.ptr(q2), flags,
                                        precision, gamma, N.ptr(flux), N.ptr(ds), N.ptr(rc, N.I32)))
    return flux, ds, rc
