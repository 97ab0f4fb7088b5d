"""ctypes bindings of the C ABI in include/titan_b200.h (libtitan_b200.so).

The shared library is built in-tree (``titan_c-_b200/build.py``); importing
this module never falls back to anything else — a missing library raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtitan_b200.so")

NV = 10
FIELDS = ("rho", "Vx", "Vy", "Vz", "p", "Bx", "By", "Bz", "Q", "rho_He")

TITAN_OK = 0
STATUS_NAMES = {0: "TITAN_OK", -1: "TITAN_EINVAL", -2: "TITAN_EMESH", -3: "TITAN_ENONFINITE", -4: "TITAN_ECUDA",
                -5: "TITAN_ETIMEOUT", -6: "TITAN_ENOMEM", -7: "TITAN_ESOLVER"}

D = ctypes.POINTER(ctypes.c_double)
I32 = ctypes.POINTER(ctypes.c_int32)
I8 = ctypes.POINTER(ctypes.c_int8)
U8 = ctypes.POINTER(ctypes.c_uint8)
I64 = ctypes.POINTER(ctypes.c_int64)


class TitanError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class TitanMesh(ctypes.Structure):
    _fields_ = [
        ("nnode", ctypes.c_int64), ("ncell", ctypes.c_int64), ("nface", ctypes.c_int64), ("nbc", ctypes.c_int64),
        ("node_xyz", D), ("cell_nodes", I32), ("cell_faces", I32), ("cell_type", I8), ("cell_tvd", U8),
        ("face_nodes", I32), ("face_cells", I32), ("face_type", I8), ("face_surf", I8), ("face_bc", I32),
        ("bc_vals", D), ("node_amp", D), ("node_phase", D),
    ]


class TitanParams(ctypes.Structure):
    _fields_ = [
        ("gamma", ctypes.c_double), ("KFL", ctypes.c_double), ("velosity_inf", ctypes.c_double),
        ("omega", ctypes.c_double), ("par_a_2", ctypes.c_double), ("par_n_H_LISM", ctypes.c_double),
        ("par_Kn", ctypes.c_double), ("beta_switch", ctypes.c_double),
        ("move", ctypes.c_int32), ("soft_fixups", ctypes.c_int32), ("method_policy", ctypes.c_int32),
        ("npassive", ctypes.c_int32), ("nh", ctypes.c_int32), ("TS_hard", ctypes.c_int32),
        ("contact_hard", ctypes.c_int32), ("flux_precision", ctypes.c_int32),
        ("tvd", ctypes.c_int32), ("snos_on_hp", ctypes.c_int32), ("bn_in_p_on_hp", ctypes.c_int32),
    ]


class TitanDevMesh(ctypes.Structure):
    """titan_dev_mesh: device pointers (as integers) for titan_step_noalloc."""
    _fields_ = [("ncell", ctypes.c_int64), ("nface", ctypes.c_int64), ("nbc", ctypes.c_int64)] + [
        (name, ctypes.c_void_p) for name in (
            "face_c0", "face_c1", "face_type", "face_surf", "face_method", "face_bc", "bc_vals", "cell_faces",
            "cell_type", "cell_tvd", "cell_center", "cell_volume", "face_center", "face_normal", "face_area",
            "face_half_dist", "hfluids")]


class TitanSurfaceParams(ctypes.Structure):
    _fields_ = [("velocity_TS", ctypes.c_double), ("velocity_HP", ctypes.c_double), ("velocity_BS", ctypes.c_double),
                ("move_TS", ctypes.c_int32), ("move_HP", ctypes.c_int32), ("move_BS", ctypes.c_int32),
                ("null_bn_on_HP", ctypes.c_int32), ("sglag_TS", ctypes.c_int32), ("sglag_HP", ctypes.c_int32),
                ("sglag_BS", ctypes.c_int32), ("hp_tail", ctypes.c_int32), ("sglag_TS_k_sphere", ctypes.c_double),
                ("sglag_HP_k_sphere", ctypes.c_double), ("sglag_BS_k", ctypes.c_double)]


class TitanRayLaw(ctypes.Structure):
    _fields_ = [("M0", ctypes.c_int32), ("M1", ctypes.c_int32), ("M11", ctypes.c_int32), ("M2", ctypes.c_int32),
                ("M3", ctypes.c_int32), ("M4", ctypes.c_int32), ("pad", ctypes.c_int32 * 2),
                ("R0", ctypes.c_double), ("R1", ctypes.c_double), ("R5", ctypes.c_double),
                ("da1", ctypes.c_double), ("da2", ctypes.c_double), ("da3", ctypes.c_double),
                ("da4", ctypes.c_double), ("da5", ctypes.c_double)]


class TitanMcParams(ctypes.Structure):
    _fields_ = [("n_H", ctypes.c_double), ("u_H", ctypes.c_double * 3), ("cp_H", ctypes.c_double),
                ("n_particles", ctypes.c_int64), ("seed", ctypes.c_uint64), ("max_cells", ctypes.c_int32),
                ("face_types", ctypes.c_int32), ("trace_out", ctypes.c_void_p)]


class TitanMcFaceDist(ctypes.Structure):
    _fields_ = [("nface", ctypes.c_int64), ("face", ctypes.c_void_p), ("side", ctypes.c_void_p),
                ("frame", ctypes.c_void_p), ("leaf_ptr", ctypes.c_void_p), ("leaf_box", ctypes.c_void_p),
                ("leaf_f", ctypes.c_void_p)]


class TitanMcFaceTally(ctypes.Structure):
    _fields_ = [("nface", ctypes.c_int64), ("face", ctypes.c_void_p), ("side", ctypes.c_void_p),
                ("frame", ctypes.c_void_p), ("leaf_ptr", ctypes.c_void_p), ("leaf_box", ctypes.c_void_p)]


class TitanMcInfo(ctypes.Structure):
    _fields_ = [("particles", ctypes.c_int64), ("lost", ctypes.c_int64), ("inflow_rate", ctypes.c_double),
                ("gpu_ms", ctypes.c_double)]


class TitanMlpTrainOpts(ctypes.Structure):
    _fields_ = [("epochs", ctypes.c_int32), ("batch", ctypes.c_int32), ("lr", ctypes.c_float),
                ("beta1", ctypes.c_float), ("beta2", ctypes.c_float), ("lr_decay", ctypes.c_float)]


MLP_NPARAM = 53776
F32 = ctypes.POINTER(ctypes.c_float)


class TitanStepInfo(ctypes.Structure):
    _fields_ = [
        ("steps_done", ctypes.c_int64), ("err_index", ctypes.c_int64), ("n_rho_floor", ctypes.c_int64),
        ("n_p_floor", ctypes.c_int64), ("status", ctypes.c_int32), ("err_kind", ctypes.c_int32),
        ("dt_next", ctypes.c_double), ("t", ctypes.c_double), ("gpu_ms", ctypes.c_double),
    ]


# Every symbol include/titan_b200.h declares, with its ctypes signature.
SIGNATURES = {
    "titan_version": ([], ctypes.c_char_p),
    "titan_last_error": ([], ctypes.c_char_p),
    "titan_create": ([ctypes.POINTER(TitanMesh), ctypes.POINTER(TitanParams), ctypes.POINTER(ctypes.c_void_p)],
                     ctypes.c_int),
    "titan_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "titan_set_face_method": ([ctypes.c_void_p, I8], ctypes.c_int),
    "titan_set_surface_motion": ([ctypes.c_void_p, ctypes.POINTER(TitanSurfaceParams), ctypes.c_int64,
                                  ctypes.c_int32, I32], ctypes.c_int),
    "titan_set_ray_law": ([ctypes.c_void_p, ctypes.POINTER(TitanRayLaw)], ctypes.c_int),
    "titan_set_mc_face_dist": ([ctypes.c_void_p, ctypes.POINTER(TitanMcFaceDist)], ctypes.c_int),
    "titan_set_mc_face_tally": ([ctypes.c_void_p, ctypes.POINTER(TitanMcFaceTally)], ctypes.c_int),
    "titan_get_mc_face_tally": ([ctypes.c_void_p, D, D, ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
    "titan_upload_state": ([ctypes.c_void_p, D], ctypes.c_int),
    "titan_download_state": ([ctypes.c_void_p, D], ctypes.c_int),
    "titan_upload_hfluids": ([ctypes.c_void_p, D], ctypes.c_int),
    "titan_set_sources": ([ctypes.c_void_p, D], ctypes.c_int),
    "titan_step": ([ctypes.c_void_p, ctypes.c_int64, D, D, ctypes.POINTER(TitanStepInfo)], ctypes.c_int),
    "titan_set_clock": ([ctypes.c_void_p, ctypes.c_double, ctypes.c_double], ctypes.c_int),
    "titan_step_async": ([ctypes.c_void_p, ctypes.c_int64], ctypes.c_int),
    "titan_get_clock": ([ctypes.c_void_p, D, D, ctypes.POINTER(TitanStepInfo)], ctypes.c_int),
    "titan_dt_copy": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32], ctypes.c_int),
    "titan_download_nodes": ([ctypes.c_void_p, D], ctypes.c_int),
    "titan_download_geometry": ([ctypes.c_void_p, D, D, D, D, D], ctypes.c_int),
    "titan_download_face_fluxes": ([ctypes.c_void_p, D], ctypes.c_int),
    "titan_get_permutation": ([ctypes.c_void_p, I32, I32, I32], ctypes.c_int),
    "titan_sfc_renumber": ([ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, D, I32, I32, I32, I32, I32],
                           ctypes.c_int),
    "titan_riemann_batch": ([ctypes.c_int64, I8, D, D, D, D, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, D, D,
                             I32], ctypes.c_int),
    "titan_mc_sources": ([ctypes.c_void_p, ctypes.POINTER(TitanMcParams), D, ctypes.POINTER(TitanMcInfo)],
                         ctypes.c_int),
    "titan_mlp_forward": ([F32, F32, F32, ctypes.c_int64, F32], ctypes.c_int),
    "titan_mlp_grad": ([F32, F32, F32, F32, F32, F32, ctypes.c_int64, F32, F32, F32], ctypes.c_int),
    "titan_mlp_train": ([F32, F32, F32, F32, F32, F32, ctypes.c_int64, ctypes.POINTER(TitanMlpTrainOpts), F32],
                        ctypes.c_int),
    "titan_get_tvd_neighbours": ([ctypes.c_void_p, I32], ctypes.c_int),
    "titan_godunov_batch": ([ctypes.c_int64, D, D, D, D, I8, ctypes.c_double, D, D, I32], ctypes.c_int),
    "titan_upload_nodes": ([ctypes.c_void_p, D], ctypes.c_int),
    "titan_read_cell_parameters": ([ctypes.c_char_p, ctypes.c_int64, ctypes.c_int64, D, D, I32, I32], ctypes.c_int),
    "titan_write_cell_parameters": ([ctypes.c_char_p, ctypes.c_int64, ctypes.c_int32, D, ctypes.c_int64, D],
                                    ctypes.c_int),
    "titan_set_closure": ([ctypes.c_void_p, F32, F32, ctypes.c_double, ctypes.c_double], ctypes.c_int),
    "titan_set_closure_fallback": ([ctypes.c_void_p, F32, F32, D], ctypes.c_int),
    "titan_closure_outside": ([ctypes.c_void_p, I64], ctypes.c_int),
    "titan_closure_fallback_from_mc": ([ctypes.c_void_p], ctypes.c_int),
    "titan_set_halo": ([ctypes.c_void_p, ctypes.c_int64, I32, ctypes.c_int64, I32], ctypes.c_int),
    "titan_set_cfl_faces": ([ctypes.c_void_p, I8], ctypes.c_int),
    "titan_pack_halo": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "titan_unpack_halo": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "titan_autotune": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_char_p], ctypes.c_int),
    "titan_set_tuning": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32], ctypes.c_int),
    "titan_set_closure_overlap": ([ctypes.c_void_p, ctypes.c_int32], ctypes.c_int),
    "titan_get_tuning": ([ctypes.c_void_p, I32, I32, I32, I32, I32], ctypes.c_int),
    "titan_stream": ([ctypes.c_void_p], ctypes.c_void_p),
    "titan_set_profiling": ([ctypes.c_void_p, ctypes.c_int32], ctypes.c_int),
    "titan_kernel_times": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_char_p), D, I64, ctypes.c_int32],
                           ctypes.c_int),
    "titan_device_bytes": ([ctypes.c_void_p], ctypes.c_int64),
    "titan_step_noalloc": ([ctypes.POINTER(TitanDevMesh), ctypes.POINTER(TitanParams), ctypes.c_double,
                            ctypes.c_void_p, ctypes.c_void_p, D, ctypes.POINTER(ctypes.c_int32), ctypes.c_void_p],
                           ctypes.c_int),
}

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded C ABI library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python titan_c-_b200/build.py` "
                               "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != TITAN_OK:
        raise TitanError(rc, lib().titan_last_error().decode(errors="replace"))


def ptr(a: np.ndarray | None, t=D):
    if a is None:
        return None
    assert a.flags.c_contiguous
    return a.ctypes.data_as(t)
