"""ctypes binding of libsht.so (the C ABI declared in include/sht.h).

The library is built in-tree (``make -C speedyweather.jl_b200/csrc``) and there is
no fallback: importing this module without the library raises ImportError.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libsht.so")

SHT_OK, SHT_EINVAL, SHT_ECUDA, SHT_ENOMEM, SHT_EUNSUPPORTED = 0, 1, 2, 3, 4
SHT_STATUS_DIAG_EXPIRED, SHT_STATUS_DIAG_FAILED = 9, 10     # device status words of sht_diag_wait_expiry
GRID_FULL_GAUSSIAN, GRID_OCTAHEDRAL_GAUSSIAN = 0, 1
PREC_FP32, PREC_BF16X3, PREC_FP16X3, PREC_BF16X5 = 0, 1, 2, 3
SHORTCUTS = {"linear": 0, "quadratic": 1, "cubic": 2, "linquadcoslat2": 3, "lincubcoslat": 4}
UNSCALE_COSLAT, ADD, FLIPSIGN, INVERSE = 1, 2, 4, 8
SYNTHESIS, ANALYSIS = 0, 1


class ShtDesc(C.Structure):
    _fields_ = [("grid", C.c_int), ("nlat_half", C.c_int), ("lmax", C.c_int), ("mmax", C.c_int),
                ("nlayers", C.c_int), ("precision", C.c_int), ("shortcut", C.c_int), ("device", C.c_int)]


class ShtInfo(C.Structure):
    _fields_ = [("npoints", C.c_int64), ("nlm", C.c_int64), ("nlat", C.c_int32), ("nlat_half", C.c_int32),
                ("nlon_max", C.c_int32), ("nfreq_max", C.c_int32), ("lmax", C.c_int32), ("mmax", C.c_int32),
                ("nlayers", C.c_int32), ("precision", C.c_int32), ("scratch_bytes", C.c_int64),
                ("table_bytes", C.c_int64)]


class ShtOp(C.Structure):
    _fields_ = [("kind", C.c_int32), ("flags", C.c_uint32), ("out", C.c_void_p), ("out2", C.c_void_p),
                ("a", C.c_void_p), ("b", C.c_void_p), ("ldc", C.c_int64), ("K", C.c_int32), ("pad", C.c_int32),
                ("radius", C.c_double)]


OP_CURL, OP_DIVERGENCE, OP_LAPLACE, OP_GRADIENT, OP_UV_FROM_VORDIV = 0, 1, 2, 3, 4
MAX_OPS = 16


class ShtBatchItem(C.Structure):
    _fields_ = [("plan", C.c_void_p), ("direction", C.c_int), ("coeffs", C.c_void_p), ("ldc", C.c_int64),
                ("grid", C.c_void_p), ("ldg", C.c_int64), ("nlayers", C.c_int), ("flags", C.c_uint)]


# name -> (restype, argtypes); every symbol the header declares
_P = C.c_void_p
_I64 = C.c_int64
SIGNATURES = {
    "sht_plan_create": (C.c_int, [C.POINTER(ShtDesc), C.POINTER(C.c_void_p)]),
    "sht_plan_destroy": (C.c_int, [_P]),
    "sht_plan_info": (C.c_int, [_P, C.POINTER(ShtInfo)]),
    "sht_plan_tables": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int32),
                                  C.POINTER(C.c_int32)]),
    "sht_synthesize": (C.c_int, [_P, _P, _I64, _P, _I64, C.c_int, C.c_uint, _P]),
    "sht_analyze": (C.c_int, [_P, _P, _I64, _P, _I64, C.c_int, C.c_uint, _P]),
    "sht_plan_set_host_chunk": (C.c_int, [_P, C.c_int]),
    "sht_synthesize_host": (C.c_int, [_P, _P, _I64, _P, _I64, C.c_int, C.c_uint, _P]),
    "sht_analyze_host": (C.c_int, [_P, _P, _I64, _P, _I64, C.c_int, C.c_uint, _P]),
    "sht_host_wait": (C.c_int, [_P, _P]),
    "sht_legendre_synthesis": (C.c_int, [_P, _P, _I64, C.c_int, _P]),
    "sht_fourier_synthesis": (C.c_int, [_P, _P, _I64, C.c_int, C.c_uint, _P]),
    "sht_fourier_analysis": (C.c_int, [_P, _P, _I64, C.c_int, _P]),
    "sht_legendre_analysis": (C.c_int, [_P, _P, _I64, C.c_int, C.c_uint, _P]),
    "sht_curl": (C.c_int, [_P, _P, _P, _P, _I64, C.c_int, C.c_uint, C.c_double, _P]),
    "sht_divergence": (C.c_int, [_P, _P, _P, _P, _I64, C.c_int, C.c_uint, C.c_double, _P]),
    "sht_uv_from_vordiv": (C.c_int, [_P, _P, _P, _P, _P, _I64, C.c_int, C.c_double, _P]),
    "sht_laplace": (C.c_int, [_P, _P, _P, _I64, C.c_int, C.c_uint, C.c_double, _P]),
    "sht_gradient": (C.c_int, [_P, _P, _P, _P, _I64, C.c_int, C.c_double, _P]),
    "sht_operators": (C.c_int, [_P, C.POINTER(ShtOp), C.c_int, _P]),
    "sht_device_status": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "sht_diag_wait_expiry": (C.c_int, [_P, C.c_int32, _P]),
    "sht_analyze_static_scratch": (C.c_int, [_P, _P, _I64, _P, _I64, C.c_int, C.c_uint, _P]),
    "sht_plan_autotune": (C.c_int, [_P, C.c_int, _P, C.POINTER(C.c_int32)]),
    "sht_plan_set_tile_columns": (C.c_int, [_P, C.c_int, C.c_int]),
    "sht_plan_set_fusion": (C.c_int, [_P, C.c_int]),
    "sht_plan_get_fusion": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "sht_plan_set_prime_stage": (C.c_int, [_P, C.c_int]),
    "sht_plan_get_prime_stage": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "sht_synthesize_adjoint": (C.c_int, [_P, _P, _I64, _P, _I64, C.c_int, C.c_uint, _P]),
    "sht_analyze_adjoint": (C.c_int, [_P, _P, _I64, _P, _I64, C.c_int, C.c_uint, _P]),
    "sht_batch_create": (C.c_int, [C.POINTER(ShtBatchItem), C.c_int, C.POINTER(C.c_void_p)]),
    "sht_batch_run": (C.c_int, [_P, _P]),
    "sht_batch_run_each": (C.c_int, [_P, _P]),
    "sht_batch_capture": (C.c_int, [_P, _P]),
    "sht_batch_launch": (C.c_int, [_P, _P]),
    "sht_batch_autotune": (C.c_int, [_P, _P, C.POINTER(C.c_int32)]),
    "sht_batch_destroy": (C.c_int, [_P]),
    "sht_matrix_create": (C.c_int, [C.POINTER(ShtDesc), C.POINTER(C.c_void_p)]),
    "sht_matrix_synthesize": (C.c_int, [_P, _P, _I64, _P, _I64, C.c_int, C.c_uint, _P]),
    "sht_matrix_analyze": (C.c_int, [_P, _P, _I64, _P, _I64, C.c_int, C.c_uint, _P]),
    "sht_matrix_device_status": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "sht_matrix_destroy": (C.c_int, [_P]),
    "sht_column_physics": (C.c_int, [_P, _P, _P, _I64, C.c_int, C.c_int, C.c_double, _P, _P, C.c_uint, _P]),
    "sht_mlp_create": (C.c_int, [C.c_int, C.c_uint64, C.c_int, C.POINTER(C.c_void_p)]),
    "sht_mlp_set_normalization": (C.c_int, [_P, _P, _P, _P, _P]),
    "sht_mlp_backward": (C.c_int, [_P, _P, _P, C.c_int, _P]),
    "sht_mlp_train_step": (C.c_int, [_P, _P, _P, C.c_int, C.c_float, _P]),
    "sht_mlp_loss": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "sht_mlp_infer": (C.c_int, [_P, _P, _P, C.c_int, _P]),
    "sht_mlp_params": (C.c_int, [_P, C.c_int, _P, _P, C.c_int]),
    "sht_column_emulate": (C.c_int, [_P, _P, _P, _P, _P, _P, _I64, C.c_int, C.c_double, C.c_double, _P, _P, C.c_uint,
                                     C.POINTER(C.c_int32), _P]),
    "sht_mlp_device_status": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "sht_mlp_destroy": (C.c_int, [_P]),
    "sht_bf16_gemm": (C.c_int, [_P, _I64, C.c_int, _P, _I64, C.c_int, _P, _I64, C.c_int, C.c_int, C.c_int, _P, _P]),
    "sht_last_error": (C.c_char_p, []),
    "sht_version": (C.c_char_p, []),
}


def load(path: str = LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(f"libsht.so not built at {path}: run `make -C speedyweather.jl_b200/csrc` "
                          "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = load()


class ShtError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libsht error {code}: {msg}")
        self.code = code


class DimensionMismatch(ValueError):
    """Raised where the reference throws DimensionMismatch (spectral_transform.jl:387-423)."""


def check(rc: int):
    if rc == SHT_OK:
        return
    msg = lib.sht_last_error().decode()
    if rc == SHT_EINVAL and "DimensionMismatch" in msg:
        raise DimensionMismatch(msg)
    raise ShtError(rc, msg)
