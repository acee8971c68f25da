"""ctypes binding of libmslr.so (the C ABI declared in include/mslr.h).

The library is loaded from this package directory.  There is no fallback:
if the shared library is missing or fails to load, importing this module
raises, so a GPU run can never silently take another path.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmslr.so")

MSLR_OK = 0
MSLR_ERR_ARG = 1
MSLR_ERR_CUDA = 2
MSLR_ERR_STATE = 3
MSLR_ERR_UNSUPPORTED = 4
MSLR_ERR_NONFINITE = 5
MSLR_ERR_NOMEM = 6

FORM_PLAIN = 0
FORM_TUNED = 1
FORM_TF32 = 2

# name -> (restype, argtypes)
_P = C.c_void_p
_I32 = C.c_int32
_I64 = C.c_int64
_D = C.c_double
_I32P = C.POINTER(C.c_int32)
SIGNATURES = {
    "mslr_abi_version": (C.c_int, []),
    "mslr_last_error": (C.c_char_p, [_P]),
    "mslr_patch_geometry": (C.c_int, [_I32P, _I32P, _I32P, _I32P, _I32P, C.POINTER(C.c_int64), _I32P]),
    "mslr_img2patches": (C.c_int, [_I32P, _I32, _I32P, _I32P, _P, _P, _P]),
    "mslr_patches2img": (C.c_int, [_I32P, _I32, _I32P, _I32P, _P, _P, _P]),
    "mslr_svst_batch_workspace": (C.c_int, [_I32, _I32, _I32, C.POINTER(C.c_size_t)]),
    "mslr_svst_batch": (C.c_int, [_I32, _I32, _I32, C.POINTER(C.c_double), _P, _P, _P, C.c_size_t,
                                  _I32, _P]),
    "mslr_create": (C.c_int, [_I32P, _I32, _I32, _I64, _I32, _I32P, _I32P, _I32, C.POINTER(_P)]),
    "mslr_destroy": (C.c_int, [_P]),
    "mslr_workspace_bytes": (C.c_int, [_P, C.POINTER(C.c_size_t)]),
    "mslr_bind": (C.c_int, [_P, _P, _P, _P, _I32, _P]),
    "mslr_sense_forward": (C.c_int, [_P, _P, _P, _P]),
    "mslr_sense_adjoint": (C.c_int, [_P, _P, _P, _P]),
    "mslr_normal_op": (C.c_int, [_P, _P, _I32, _P, _I32, _P]),
    "mslr_set_graph": (C.c_int, [_P, _I32]),
    "mslr_set_lambdas": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "mslr_autotune": (C.c_int, [_P, _P]),
    "mslr_get_tuning": (C.c_int, [_P, C.POINTER(_I32), _I32, C.POINTER(_I32)]),
    "mslr_sos_normalize": (C.c_int, [_I32P, _I32, _P, _P, _P]),
    "mslr_sampling": (C.c_int, [_I32P, _I32, _I32, _P, C.POINTER(_I64), _P, _P, _I64, _P]),
    "mslr_prepare": (C.c_int, [_P, _P, _P, _P, _P, _P, C.POINTER(C.c_double), _P]),
    "mslr_get_lambdas": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "mslr_pogm_grad": (C.c_int, [_P, _P, _I32, C.c_double, C.c_double, C.c_double, _P,
                                 C.POINTER(C.c_double), C.POINTER(C.c_double), _P, _P]),
    "mslr_cost": (C.c_int, [_P, _P, _I32, C.POINTER(C.c_double), C.POINTER(C.c_double), _P]),
    "mslr_normal_op_profile": (C.c_int, [_P, _P, _I32, _P, _P, C.POINTER(C.c_double),
                                         C.POINTER(C.c_int64)]),
    "mslr_patch_svst": (C.c_int, [_P, _I32, _D, _P, _P, _P]),
    "mslr_init_x0": (C.c_int, [_P, _P, _P]),
    "mslr_pogm_run": (C.c_int, [_P, _P, _I32, _D, _D, _D, C.POINTER(C.c_uint8), _P]),
    "mslr_pogm_begin": (C.c_int, [_P, _P, _I32, _D, _D, _D, _P]),
    "mslr_pogm_step": (C.c_int, [_P, _P, _P]),
    "mslr_pogm_restarts": (C.c_int, [_P, C.POINTER(C.c_uint8), _P]),
    "mslr_launch_count": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "mslr_power_iter": (C.c_int, [_P, _I32, _D, C.POINTER(C.c_double), _I32P, _P]),
    "mslr_pogm_run_costs": (C.c_int, [_P, _P, _I32, _D, _D, _D, C.POINTER(C.c_uint8),
                                      C.POINTER(C.c_double), C.POINTER(C.c_double), _P]),
    "mslr_pogm_run_options": (C.c_int, [_P, _P, _I32, _D, _D, _I32, _I32, _D, _D,
                                        C.POINTER(C.c_uint8), _P]),
    "mslr_sync": (C.c_int, [_P, _P]),
    "mslr_set_wait_limit": (C.c_int, [_P, _I64]),
    "mslr_fp32_peak": (C.c_int, [C.POINTER(C.c_double), _P]),
    "mslr_pogm_step_local": (C.c_int, [_P, _P, _P, _P, _P]),
    "mslr_patch_svst_lambdas": (C.c_int, [_P, _I32, C.POINTER(C.c_double), _P, _P, _P]),
    "mslr_patch_nucnorm": (C.c_int, [_P, _I32, C.POINTER(C.c_double), _P, C.POINTER(C.c_double), _P]),
    "mslr_pogm_step_decide": (C.c_int, [_P, _P, _P]),
    "mslr_pogm_scalars": (C.c_int, [_P, C.POINTER(C.c_double), _P]),
    "mslr_patch_gram": (C.c_int, [_P, _I32, _P, _P, _P]),
    "mslr_patch_svst_gram": (C.c_int, [_P, _I32, _D, _P, _P, _P, _P]),
    "mslr_svst_batch_noalloc": (C.c_int, [_I32, _I32, _I32, C.POINTER(C.c_double), _P, _P, _P]),
}


class MSLRError(RuntimeError):
    """Raised for any non-zero status returned by libmslr."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[mslr status {code}] {msg}")
        self.code = code


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libmslr.so not built at {LIB_PATH}; run mslr-recon_b200/build_lib.py")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.mslr_abi_version() != 1:
        raise ImportError("libmslr ABI version mismatch")
    return lib


lib = _load()


def check(rc: int, ctx=None) -> None:
    """Raise MSLRError (ValueError for argument errors) on a non-zero status."""
    if rc == MSLR_OK:
        return
    msg = lib.mslr_last_error(ctx)
    msg = msg.decode() if msg else ""
    if rc == MSLR_ERR_ARG:
        raise ValueError(f"[mslr status {rc}] {msg}")
    raise MSLRError(rc, msg)


def i32arr(vals) -> C.Array:
    vals = [int(v) for v in vals]
    return (C.c_int32 * len(vals))(*vals)
