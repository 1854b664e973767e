"""ctypes binding of libparalanczos_b200.so (the C ABI in include/paralanczos.h).

The library is the product: nothing here computes anything itself.  If the
shared object is missing the import fails loudly (there is no fallback path).
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libparalanczos_b200.so")

PL_OK, PL_EINVAL, PL_ECUDA, PL_ENOMEM, PL_ENOTSUP, PL_ETIMEDOUT, PL_EBUSY = range(7)
PL_SET_BREAKDOWN, PL_SET_NONFINITE, PL_SET_BAD_INDEX, PL_SET_BAD_K = 1, 2, 4, 8
PL_FORM_BATCHED, PL_FORM_PLAIN = 0, 1
PL_KMAX = 512

_vp = C.c_void_p
_ll = C.c_longlong
_i = C.c_int
_d = C.c_double

# name -> (restype, argtypes); every symbol include/paralanczos.h declares
SIGNATURES = {
    "pl_version": (_i, []),
    "pl_status_string": (C.c_char_p, [_i]),
    "pl_last_cuda_error": (_i, []),
    "pl_solve": (_i, [_vp, _i, _ll, _vp, _vp, _ll, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "pl_solve_host": (_i, [_vp, _i, _ll, _vp, _vp, _ll, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "pl_solve_noalloc": (_i, [_vp, _i, _ll, _vp, _ll, _i, _vp, _vp, _vp, _vp, _vp]),
    "pl_gen_sets": (_i, [C.c_ulonglong, _ll, _ll, _i, _i, _vp, _vp]),
    "pl_gather_blocks": (_i, [_vp, _i, _ll, _vp, _ll, _i, _vp, _vp, _vp]),
    "pl_gen_stream_host": (_ll, [C.c_ulonglong, _ll, _ll, _i, _i, _i, _i, _vp, _vp]),
    "pl_convert_f64_f32": (_i, [_vp, _vp, _ll, _vp]),
    "pl_dropin_cache_stats": (None, [C.POINTER(_ll), C.POINTER(_ll)]),
    "pl_calculate_subeigs3": (_i, [_vp, _i, _i, _vp, _vp, _vp, _i]),
    "pl_calculate_subeigs": (_i, [_vp, _i, _vp, _vp, _vp, _i]),
    "pl_calculate_subeigs2": (_i, [_vp, _i, _i, _vp, _vp, _vp, _i]),
    "pl_calculate_eigs": (_i, [_vp, _i, _vp, _vp]),
    "pl_tune_set": (_i, [_i, _i]),
    "pl_tune_get": (_i, [_i]),
    "pl_tune_describe": (_i, [_i, _i, C.c_char_p, _i]),
    "pl_num_bins": (_i, []),
    "pl_bin_kmax": (_i, [_i]),
    "pl_fp32_peak": (_i, [C.POINTER(_d), _vp]),
    "pl_gather_peak": (_i, [C.POINTER(_d), _vp]),
    "pl_release": (_i, []),
    "pl_gram_prep_bytes": (_ll, [_i, _i]),
    "pl_gram_prepare": (_i, [_vp, _ll, _i, _i, _vp, _vp]),
    "pl_gram_blocks": (_i, [_vp, _i, _i, _vp, _ll, _i, _vp, _vp, _vp]),
    "pl_solve_gram": (_i, [_vp, _i, _i, _vp, _ll, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "pl_serve_create": (_i, [_ll, _ll, _i, C.POINTER(_vp)]),
    "pl_serve_add_matrix": (_i, [_vp, _vp, _i, _ll, C.POINTER(_i)]),
    "pl_serve_submit": (_i, [_vp, _i, _vp, _ll, _i, C.POINTER(_ll)]),
    "pl_serve_wait": (_i, [_vp, _ll, _d, _vp, _vp, _vp, _vp, C.POINTER(_d)]),
    "pl_serve_stats": (_i, [_vp, C.POINTER(_d), _i]),
    "pl_serve_reset_stats": (_i, [_vp]),
    "pl_serve_destroy": (_i, [_vp]),
    "pl_launch_reference_kernel": (_i, [C.c_char_p, C.c_uint, C.c_uint, C.c_uint, C.POINTER(_vp), _vp]),
}

_lib = None


class PLError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = f"{where}: {status_string(status)} (status {status})"
        if status == PL_ECUDA and _lib is not None:
            msg += f", cudaError {_lib.pl_last_cuda_error()}"
        super().__init__(msg)
        self.status = status


def lib():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m paralanczos_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
        # launch shapes chosen by the autotuner for this GPU, when present
        from . import autotune
        autotune.apply(lib=L)
    return _lib


def status_string(s: int) -> str:
    if _lib is None:
        return {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory",
                4: "not supported", 5: "timed out", 6: "busy"}.get(s, "unknown status")
    return _lib.pl_status_string(s).decode()


def check(status: int, where: str) -> None:
    if status != PL_OK:
        raise PLError(status, where)
