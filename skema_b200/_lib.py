"""ctypes binding of the C ABI in ``include/skema_c.h``.

The CUDA library ``libskema_b200.so`` is loaded from this package directory.
There is no fallback: if the library is missing or cannot be loaded, every
entry point raises ``SkemaError``.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libskema_b200.so")

# status codes (skema_status)
OK, EINVAL, ENOMEM, ECUDA, ENOTPD, ETIMEOUT, ESTATE, EUNSUPPORTED, ENOKERNEL, ECOLLECTIVE = range(10)
STATUS_NAMES = {
    OK: "OK", EINVAL: "EINVAL", ENOMEM: "ENOMEM", ECUDA: "ECUDA", ENOTPD: "ENOTPD",
    ETIMEOUT: "ETIMEOUT", ESTATE: "ESTATE", EUNSUPPORTED: "EUNSUPPORTED", ENOKERNEL: "ENOKERNEL",
    ECOLLECTIVE: "ECOLLECTIVE",
}
MAP_GAUSS, MAP_SPARSE_SIGN = 0, 1
KERNEL_NONE, KERNEL_GAUSSRBF = 0, 1
PREC_FP32, PREC_BF16, PREC_FP8 = 0, 1, 2
SPD_NYSTROM, SPD_REFERENCE_STEPS = 0, 1
UPSILON, OMEGA, PHI, PSI = 0, 1, 2, 3
COL_MAJOR, ROW_MAJOR = 0, 1
MEM_DEVICE, MEM_HOST = 0, 1
SKETCH_X, SKETCH_Y, SKETCH_Z = 0, 1, 2


class SkemaError(RuntimeError):
    """A non-OK status from the C ABI (the shim's std::runtime_error)."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


class Params(C.Structure):
    """``skema_params``: the sketch fields of Skema::AlgParams."""

    _fields_ = [
        ("matrix_m", C.c_int64),
        ("matrix_n", C.c_int64),
        ("rank", C.c_int64),
        ("sketch_range", C.c_int64),
        ("sketch_core", C.c_int64),
        ("window", C.c_int64),
        ("sketch_eta", C.c_double),
        ("sketch_nu", C.c_double),
        ("seeds", C.c_int32 * 4),
        ("dim_redux", C.c_int32),
        ("issparse", C.c_int32),
        ("issymmetric", C.c_int32),
        ("force_three_sketch", C.c_int32),
        ("kernel_func", C.c_int32),
        ("kernel_gamma", C.c_double),
        ("precision", C.c_int32),
        ("device", C.c_int32),
        ("spd_approx", C.c_int32),
    ]


class Crs(C.Structure):
    """``skema_crs``: a CRS matrix returned by skema_read_crs."""

    _fields_ = [("nrow", C.c_int64), ("ncol", C.c_int64), ("nnz", C.c_int64),
                ("rowptr", C.POINTER(C.c_int64)), ("col", C.POINTER(C.c_int32)), ("val", C.POINTER(C.c_double))]


# skema_allreduce_fn: int (*)(double* buf, int64_t count, void* user)
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_void_p)


class Dense(C.Structure):
    """``skema_dense``: a column-major matrix returned by skema_read_dense."""

    _fields_ = [("nrow", C.c_int64), ("ncol", C.c_int64), ("data", C.POINTER(C.c_double))]


class MatF(C.Structure):
    """``skema_matf``: a dense FP32 operand of the map products."""

    _fields_ = [("p", C.c_void_p), ("rows", C.c_int64), ("cols", C.c_int64), ("ld", C.c_int64),
                ("layout", C.c_int32)]


class CsrF(C.Structure):
    """``skema_csrf``: a CSR FP32 operand of the map products."""

    _fields_ = [("rowptr", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p), ("rows", C.c_int64),
                ("cols", C.c_int64)]


_P = C.c_void_p
_I64 = C.c_int64
_I32 = C.c_int32
_D = C.c_double

# name -> (restype, argtypes)
SIGNATURES = {
    "skema_params_init": (C.c_int, [C.POINTER(Params)]),
    "skema_create": (C.c_int, [C.POINTER(Params), C.POINTER(_P)]),
    "skema_destroy": (C.c_int, [_P]),
    "skema_last_error": (C.c_char_p, [_P]),
    "skema_get_dims": (C.c_int, [_P, C.POINTER(_I64), C.POINTER(_I64), C.POINTER(_I32)]),
    "skema_reset": (C.c_int, [_P]),
    "skema_linear_update_dense": (C.c_int, [_P, _P, _I64, _I32, _I64, _I64, _I32]),
    "skema_linear_update_csr": (C.c_int, [_P, _P, _P, _P, _I64, _I64, _I32]),
    "skema_linear_update_rbf": (C.c_int, [_P, _P, _I64, _I32, _I64, _I64, _I64, _I64, _I32]),
    "skema_low_rank_approx": (C.c_int, [_P, _P, _P, _P, _I32]),
    "skema_low_rank_approx_rows": (C.c_int, [_P, _I64, _I64, _P, _P, _P, _P, _P, _I32]),
    "skema_residuals_begin": (C.c_int, [_P, _P, _P, _P, _I32]),
    "skema_set_keep_factors": (C.c_int, [_P, _I32]),
    "skema_residuals_update_dense": (C.c_int, [_P, _P, _I64, _I32, _I64, _I64, _I32]),
    "skema_residuals_update_csr": (C.c_int, [_P, _P, _P, _P, _I64, _I64, _I32]),
    "skema_residuals_update_rbf": (C.c_int, [_P, _P, _I64, _I32, _I64, _I64, _I64, _I64, _I32]),
    "skema_residuals_finish": (C.c_int, [_P, _P, _I32]),
    "skema_get_sketch": (C.c_int, [_P, _I32, _P, _I64, _I32, _I32]),
    "skema_set_sketch": (C.c_int, [_P, _I32, _P, _I64, _I32, _I32]),
    "skema_map_info": (C.c_int, [_P, _I32, C.POINTER(_I64), C.POINTER(_I64), C.POINTER(_I32), C.POINTER(_I32)]),
    "skema_map_export": (C.c_int, [_P, _I32, _P, _P]),
    "skema_map_import": (C.c_int, [_P, _I32, _P, _P]),
    "skema_rbf_sketch_fwd": (C.c_int, [_P, _P, _I64, _I64, _D, _P, _I64, _P]),
    "skema_rbf_sketch_vjp": (C.c_int, [_P, _P, _I64, _I64, _D, _P, _I64, _P, _P, _P]),
    "skema_rbf_sketch_fwd_noalloc": (C.c_int, [_P, _P, _I64, _I64, _D, _P, _I64, _P]),
    "skema_synchronize": (C.c_int, [_P]),
    "skema_set_stream": (C.c_int, [_P, _P]),
    "skema_get_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "skema_set_wait_limit": (C.c_int, [_P, _I64]),
    "skema_set_workspace_limit": (C.c_int, [_P, _I64]),
    "skema_launch_count": (_I64, [_P]),
    "skema_timing_enable": (C.c_int, [_P, _I32]),
    "skema_timing_get": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_double), C.POINTER(_I64)]),
    "skema_dimredux_create": (C.c_int, [_I32, _I64, _I64, _I32, _I32, C.POINTER(_P)]),
    "skema_dimredux_destroy": (C.c_int, [_P]),
    "skema_dimredux_last_error": (C.c_char_p, [_P]),
    "skema_dimredux_export": (C.c_int, [_P, _P, _P]),
    "skema_dimredux_lmap": (C.c_int, [_P, _D, C.POINTER(MatF), _D, C.c_char, C.c_char, _I64, _I64,
                                      C.POINTER(MatF), _I32]),
    "skema_dimredux_rmap": (C.c_int, [_P, _D, C.POINTER(MatF), _D, C.c_char, C.c_char, _I64, _I64,
                                      C.POINTER(MatF), _I32]),
    "skema_dimredux_lmap_csr": (C.c_int, [_P, _D, C.POINTER(CsrF), _D, C.c_char, C.c_char, _I64, _I64,
                                          C.POINTER(MatF), _I32]),
    "skema_dimredux_rmap_csr": (C.c_int, [_P, _D, C.POINTER(CsrF), _D, C.c_char, C.c_char, _I64, _I64,
                                          C.POINTER(MatF), _I32]),
    "skema_read_crs": (C.c_int, [C.c_char_p, C.POINTER(Crs)]),
    "skema_crs_free": (None, [C.POINTER(Crs)]),
    "skema_read_dense": (C.c_int, [C.c_char_p, C.POINTER(Dense)]),
    "skema_dense_free": (None, [C.POINTER(Dense)]),
    "skema_write_crs": (C.c_int, [C.c_char_p, C.POINTER(Crs)]),
    "skema_read_crs_rows": (C.c_int, [C.c_char_p, _I64, _I64, C.POINTER(Crs)]),
    "skema_update_from_file": (C.c_int, [_P, C.c_char_p, _I64, _I64]),
}

_lib = None


def load(path: str | None = None) -> C.CDLL:
    """Load the CUDA library (once) and attach the C signatures."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise SkemaError(ENOKERNEL, f"CUDA library not built: {p} (run python -m skema_b200.build)")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(status: int, ctx=None) -> None:
    if status != OK:
        msg = load().skema_last_error(ctx)
        raise SkemaError(status, msg.decode() if msg else "")


def default_params() -> Params:
    p = Params()
    check(load().skema_params_init(C.byref(p)))
    return p
