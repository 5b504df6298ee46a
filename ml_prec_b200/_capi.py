"""ctypes binding of the C ABI in include/mlp_b200.h.

The shared library is built in-tree (ml_prec_b200/lib/libmlp_b200.so); if it is
missing this module raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libmlp_b200.so")

u32p = C.POINTER(C.c_uint32)
f64p = C.POINTER(C.c_double)

# Every symbol include/mlp_b200.h declares (checked by the CPU test suite).
EXPORTS = [
    "mlp_last_error", "mlp_version", "mlp_device_count", "mlp_set_device",
    "mlp_matrix_create", "mlp_matrix_create_spe", "mlp_matrix_destroy", "mlp_matrix_size",
    "mlp_matrix_download", "mlp_spmv", "mlp_spmv_host",
    "mlp_prec_create", "mlp_prec_destroy", "mlp_prec_apply", "mlp_prec_apply_host", "mlp_prec_nlevels",
    "mlp_prec_level_info", "mlp_prec_level_export", "mlp_prec_bytes_per_apply", "mlp_prec_profile",
    "mlp_prec_timeline", "mlp_pcg_timeline",
    "mlp_pcg", "mlp_pcg_device", "mlp_pcg_device_x0", "mlp_matrix_grad_logk", "mlp_pcg_device_noalloc",
    "mlp_launch_count", "mlp_generate_x0", "mlp_cheb_solve", "mlp_cheb_solve_device", "mlp_ensemble_create", "mlp_ensemble_solve", "mlp_ensemble_destroy",
    "mlp_ensemble_gradient_create",
]


class PrecCfg(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("nq", C.c_uint32), ("q", f64p),
        ("nniter", C.c_uint32), ("niter", u32p),
        ("coarse_n", C.c_uint32), ("max_levels", C.c_uint32), ("degree_max", C.c_uint32),
        ("order", C.c_int32), ("use_tails", C.c_int32),
        ("nsigma", C.c_uint32), ("sigma", f64p),
        ("nncheb", C.c_uint32), ("ncheb", u32p),
        ("fp32", C.c_int32),
        ("autotune", C.c_int32),
        ("neps", C.c_uint32), ("level_eps", f64p),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("niter", C.c_uint32), ("napply", C.c_uint32),
        ("init_norm", C.c_double), ("final_norm", C.c_double), ("final_rel", C.c_double),
        ("t_solve_ms", C.c_double), ("t_setup_ms", C.c_double),
    ]


class LevelInfo(C.Structure):
    _fields_ = [
        ("N", C.c_uint32), ("nnz", C.c_uint32), ("M", C.c_uint32), ("Md", C.c_uint32), ("n", C.c_uint32),
        ("niter", C.c_uint32), ("ncheb", C.c_uint32), ("direct", C.c_int32),
        ("q", C.c_double), ("alpha", C.c_double), ("beta", C.c_double), ("lmin", C.c_double),
        ("lmax", C.c_double),
        ("L_nnz", C.c_uint32), ("U_nnz", C.c_uint32),
        ("nwave_l", C.c_uint32), ("nwave_u", C.c_uint32),
        ("P1_nnz", C.c_uint32), ("G_nnz", C.c_uint32),
        ("eps", C.c_double),
    ]


class MlpError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None


def lib():
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m ml_prec_b200.build` first")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.mlp_last_error.restype = C.c_char_p
        L.mlp_matrix_create.argtypes = [C.c_uint32, u32p, u32p, f64p, C.POINTER(vp)]
        L.mlp_matrix_create_spe.argtypes = [C.c_uint32] * 3 + [f64p] * 3 + [C.c_double, C.c_int32,
                                                                           C.POINTER(vp), f64p]
        L.mlp_matrix_destroy.argtypes = [vp]
        L.mlp_matrix_size.argtypes = [vp, u32p, u32p]
        L.mlp_matrix_download.argtypes = [vp, u32p, u32p, f64p]
        L.mlp_spmv.argtypes = [vp, vp, vp, vp]
        L.mlp_spmv_host.argtypes = [vp, f64p, f64p]
        L.mlp_prec_create.argtypes = [vp, C.POINTER(PrecCfg), C.POINTER(vp)]
        L.mlp_prec_destroy.argtypes = [vp]
        L.mlp_prec_apply.argtypes = [vp, vp, vp, vp]
        L.mlp_prec_apply_host.argtypes = [vp, f64p, f64p]
        L.mlp_prec_nlevels.argtypes = [vp, u32p]
        L.mlp_prec_level_info.argtypes = [vp, C.c_uint32, C.POINTER(LevelInfo)]
        L.mlp_prec_level_export.argtypes = [vp, C.c_uint32, u32p, u32p, u32p, f64p, u32p, u32p, f64p,
                                             u32p, u32p, f64p, f64p]
        L.mlp_prec_bytes_per_apply.argtypes = [vp, C.POINTER(C.c_uint64)]
        L.mlp_prec_profile.argtypes = [vp, C.c_uint32, C.c_uint32, u32p, f64p, C.POINTER(C.c_uint64), C.c_char_p,
                                       C.c_uint32]
        L.mlp_prec_timeline.argtypes = [vp, C.c_uint32, C.c_uint32, u32p, f64p]
        L.mlp_pcg_timeline.argtypes = [vp, vp, vp, vp, C.c_double, C.c_int32, C.c_uint32, u32p, f64p, C.c_char_p,
                                       C.c_uint32]
        L.mlp_pcg.argtypes = [vp, f64p, vp, f64p, C.c_double, C.c_uint32, C.c_int32, C.POINTER(Stats)]
        L.mlp_pcg_device.argtypes = [vp, vp, vp, vp, C.c_double, C.c_uint32, C.c_int32, C.POINTER(Stats), vp]
        L.mlp_generate_x0.argtypes = [f64p, C.c_uint32]
        L.mlp_cheb_solve.argtypes = [vp, f64p, vp, f64p, C.c_double, C.c_double, C.c_double, C.c_uint32,
                                     C.POINTER(Stats)]
        L.mlp_cheb_solve_device.argtypes = [vp, vp, vp, vp, C.c_double, C.c_double, C.c_double, C.c_uint32,
                                            C.POINTER(Stats), vp]
        L.mlp_pcg_device_noalloc.argtypes = [vp, vp, vp, vp, C.c_double, C.c_uint32, C.c_int32,
                                             C.POINTER(Stats), vp]
        L.mlp_launch_count.argtypes = [C.POINTER(C.c_uint64)]
        L.mlp_pcg_device_x0.argtypes = [vp, vp, vp, vp, C.c_double, C.c_uint32, C.c_int32, C.c_int32,
                                        C.POINTER(Stats), vp]
        L.mlp_matrix_grad_logk.argtypes = [vp, vp, vp, vp, vp]
        L.mlp_ensemble_create.argtypes = [C.c_uint32, C.POINTER(vp), C.c_int32, C.c_int32, C.POINTER(vp)]
        L.mlp_ensemble_solve.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.c_double, C.c_uint32,
                                         C.POINTER(Stats), C.POINTER(C.c_double), vp]
        L.mlp_ensemble_destroy.argtypes = [vp]
        L.mlp_ensemble_gradient_create.argtypes = [C.c_uint32, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), u32p,
                                                   C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                                                   C.c_int32, C.POINTER(vp)]
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        raise MlpError(rc, lib().mlp_last_error().decode(errors="replace"))


def ptr(a, t):
    return a.ctypes.data_as(t)
