"""ctypes binding of libafid_gpu.so (the C-ABI declared in include/afid_gpu.h).

There is no fallback: if the shared library is missing or cannot be loaded,
``lib()`` raises.  Build it with ``python -m afid_b200.build``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libafid_gpu.so")

AFID_OK = 0
STATUS_HELD = 1          # afid_box_scalars.status of a box on hold (not an error)
STATUS_DEVICE_TIMEOUT = 990   # a transform's tile copy did not complete within the wait limit
ERRORS = {-1: "AFID_EINVAL", -2: "AFID_ENOMEM", -3: "AFID_ECUDA", -4: "AFID_ENOBOX",
          -5: "AFID_EFFT", -6: "AFID_ESIZE"}

FIELDS = {"vx": 0, "vy": 1, "vz": 2, "temp": 3, "pr": 4, "rux": 5, "ruy": 6, "ruz": 7,
          "rutemp": 8, "dph": 9, "qcap": 10, "dq": 11, "hro": 12, "rhs": 13, "wall": 14}

# every symbol include/afid_gpu.h declares
EXPORTS = [
    "afid_version", "afid_last_error", "afid_ctx_create", "afid_ctx_destroy",
    "afid_ctx_set_stream", "afid_ctx_stream", "afid_ctx_synchronize", "afid_make_grid",
    "afid_box_device_bytes", "afid_box_add", "afid_box_remove", "afid_box_upload",
    "afid_box_download", "afid_box_reset", "afid_box_get_scalars", "afid_box_history",
    "afid_box_upload_async", "afid_box_download_async", "afid_boxes_get_scalars",
    "afid_step_graph_kernels", "afid_boxes_get_scalars_async", "afid_ctx_set_split_sets",
    "afid_time_marcher_begin_substep", "afid_explicit_terms_vx", "afid_explicit_terms_vy",
    "afid_explicit_terms_vz", "afid_explicit_terms_temp", "afid_implicit_and_update_vx",
    "afid_implicit_and_update_vy", "afid_implicit_and_update_vz",
    "afid_implicit_and_update_temp", "afid_calc_local_divergence",
    "afid_solve_pressure_correction", "afid_correct_velocity", "afid_correct_pressure",
    "afid_calc_max_cfl", "afid_check_divergence", "afid_calc_plate_nu", "afid_step",
    "afid_step_graph", "afid_substep", "afid_step_profiled",
    "afid_solve_pressure_correction_noalloc", "afid_box_set_tuning",
    "afid_global_quantities", "afid_calc_stats", "afid_calc_dissipation_nu", "afid_box_get_stats",
    "afid_box_reset_stats", "afid_slab_locations", "afid_slab_dump", "afid_box_set_time",
    "afid_box_interp_field", "afid_box_set_stop", "afid_box_resume",
    "afid_box_test_skip_z_copies",
]

STATS = ["vx_me", "vy_me", "vz_me", "temp_me", "vx_rms", "vy_rms", "vz_rms", "temp_rms", "tempvx_me",
         "disste", "dissth"]

KERNELS = ["diag", "finalize", "prep", "explicit_fwd", "implicit_bwd", "fft_y_fwd", "fft_z_fwd",
           "poisson_x", "fft_z_inv", "fft_y_inv", "correct", "plate_nu", "divergence"]


class BoxParams(C.Structure):
    _fields_ = [
        ("nxm", C.c_int), ("nym", C.c_int), ("nzm", C.c_int), ("nsst", C.c_int),
        ("alx3", C.c_double), ("ylen", C.c_double), ("zlen", C.c_double),
        ("ray", C.c_double), ("pra", C.c_double),
        ("inslws", C.c_int), ("inslwn", C.c_int),
        ("tempbp", C.c_double), ("temptp", C.c_double),
        ("dt", C.c_double), ("idtv", C.c_int),
        ("cflmax", C.c_double), ("dtmin", C.c_double), ("dtmax", C.c_double),
        ("vlim", C.c_double), ("resid", C.c_double),
    ]


class GlobalQ(C.Structure):
    _fields_ = [
        ("nu_vol", C.c_double), ("vmax", C.c_double * 3), ("tempm", C.c_double),
        ("tempmax", C.c_double), ("tempmin", C.c_double), ("vz_rms", C.c_double),
        ("vy_rms", C.c_double), ("vx_rms", C.c_double), ("vel_rms", C.c_double),
    ]


class BoxScalars(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("time", C.c_double), ("cfl", C.c_double), ("cfl_used", C.c_double),
        ("divmax", C.c_double), ("vmax", C.c_double * 3), ("nu_bot", C.c_double),
        ("nu_top", C.c_double), ("ntime", C.c_int), ("status", C.c_int),
    ]


class StepRecord(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("time", "dt", "cfl_used", "divmax", "nu_bot", "nu_top", "vmax_y", "vmax_z")]


class AfidError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_LIB = None


def lib(path: str | None = None) -> C.CDLL:
    """Load (once) and return the library; raises if it is absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"libafid_gpu.so not found at {p}: build it with "
                           "`python -m afid_b200.build` (there is no CPU fallback)")
    L = C.CDLL(p)
    vp, i, d, dp = C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    sig = {
        "afid_version": ([], i), "afid_last_error": ([], C.c_char_p),
        "afid_ctx_create": ([C.POINTER(vp), i], i), "afid_ctx_destroy": ([vp], i),
        "afid_ctx_set_stream": ([vp, vp], i), "afid_ctx_stream": ([vp], vp),
        "afid_ctx_synchronize": ([vp], i),
        "afid_make_grid": ([i, i, d, d, dp], i),
        "afid_box_device_bytes": ([C.POINTER(BoxParams)], C.c_size_t),
        "afid_box_add": ([vp, C.POINTER(BoxParams), dp, ip], i),
        "afid_box_remove": ([vp, i], i),
        "afid_box_upload": ([vp, i, i, dp], i), "afid_box_download": ([vp, i, i, dp], i),
        "afid_box_upload_async": ([vp, i, i, dp], i), "afid_box_download_async": ([vp, i, i, dp], i),
        "afid_boxes_get_scalars": ([vp, ip, i, C.POINTER(BoxScalars)], i),
        "afid_step_graph_kernels": ([vp, ip, i, ip], i),
        "afid_boxes_get_scalars_async": ([vp, ip, i, C.POINTER(BoxScalars)], i),
        "afid_ctx_set_split_sets": ([vp, i], i),
        "afid_box_reset": ([vp, i, d], i),
        "afid_box_get_scalars": ([vp, i, C.POINTER(BoxScalars)], i),
        "afid_box_history": ([vp, i, C.POINTER(StepRecord), i], i),
        "afid_time_marcher_begin_substep": ([vp, i, i], i),
        "afid_calc_max_cfl": ([vp, i, dp], i), "afid_check_divergence": ([vp, i, dp], i),
        "afid_calc_plate_nu": ([vp, i, dp, dp], i),
        "afid_step": ([vp, ip, i, i], i), "afid_step_graph": ([vp, ip, i, i], i),
        "afid_substep": ([vp, ip, i, i], i),
        "afid_step_profiled": ([vp, ip, i, i, dp, ip, i], i),
        "afid_solve_pressure_correction_noalloc": ([vp, i, i, i, dp, d, d, d, vp, ip], i),
        "afid_box_set_tuning": ([vp, i, i, i, i], i),
        "afid_global_quantities": ([vp, i, C.POINTER(GlobalQ)], i),
        "afid_calc_stats": ([vp, i], i),
        "afid_calc_dissipation_nu": ([vp, i, dp, dp], i),
        "afid_box_get_stats": ([vp, i, dp, ip], i),
        "afid_box_reset_stats": ([vp, i], i),
        "afid_slab_locations": ([i, dp, dp, ip], i),
        "afid_slab_dump": ([vp, i, ip, i, dp], i),
        "afid_box_set_time": ([vp, i, d], i),
        "afid_box_interp_field": ([vp, i, i, dp, i, i, i, i, d, i, d], i),
        "afid_box_set_stop": ([vp, i, i, d, d], i), "afid_box_resume": ([vp, i], i),
        "afid_box_test_skip_z_copies": ([vp, i, i, C.c_uint], i),
    }
    for name in ("explicit_terms_vx", "explicit_terms_vy", "explicit_terms_vz",
                 "explicit_terms_temp", "implicit_and_update_vx", "implicit_and_update_vy",
                 "implicit_and_update_vz", "implicit_and_update_temp",
                 "calc_local_divergence", "solve_pressure_correction", "correct_velocity",
                 "correct_pressure"):
        sig["afid_" + name] = ([vp, i], i)
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _LIB = L
    return L


def check(rc: int) -> int:
    if rc < 0:
        msg = lib().afid_last_error()
        raise AfidError(rc, msg.decode() if msg else "")
    return rc


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))
