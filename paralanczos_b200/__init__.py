"""paralanczos_b200 -- B200-native (sm_100a) batched subset-Lanczos eigenvalues.

Eigenvalues of many principal submatrices A[S,S] of one symmetric matrix, and
their restricted-isometry constants delta_k, computed by hand-written CUDA in
libparalanczos_b200.so behind a C ABI (include/paralanczos.h).  A drop-in for
the host API of ParaLanczos v0.21 (ParaLanczos.h).
"""
from .api import (  # noqa: F401
    calculate_eigs,
    calculate_subeigs,
    calculate_subeigs2,
    calculate_subeigs3,
    bin_kmax,
    fp32_peak,
    gen_sets,
    gen_stream_host,
    num_bins,
    release,
    solve,
    solve_host,
    tune_describe,
    tune_get,
    tune_set,
)
from ._lib import PLError, lib  # noqa: F401

__version__ = "1.0"
