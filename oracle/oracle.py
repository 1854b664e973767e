"""ctypes front end of the CPU oracle (oracle/pl_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference arm of bench.py.  The product package never imports it.

It exposes
  * the FP64 restatement of the reference's per-set path (KER2 Lanczos,
    ParaLanczos.cu:1285-1374, all-ones start; TQLRAT ParaLanczos.cu:32-189;
    DET_TRIDIAG ParaLanczos.cu:243-269), single-set and OpenMP batch;
  * the reference's own TQLRAT/DET_TRIDIAG compiled from its source into
    oracle/_ref/libplref.so (when built), to pin the restatement;
  * FP64 LAPACK dsyev truth through scipy;
  * the counter-based index-set generator (C twin of the device generator);
  * the FP64 Sturm-count bisection restated for checking the device bisection.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libplref.so")

_lib = None
_ref = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_longlong)


def build() -> None:
    """Build liboracle.so (and oracle/_ref when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    subprocess.run(["python3", os.path.join(HERE, "build_ref.py")], check=True, stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
                os.path.join(HERE, "pl_oracle.c")):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_tqlrat.argtypes = [C.c_int, _dp, _dp]
        L.orc_tqlrat.restype = C.c_int
        L.orc_det_tridiag.argtypes = [C.c_int, _dp, _dp]
        L.orc_det_tridiag.restype = C.c_double
        L.orc_ker2_lanczos.argtypes = [_dp, C.c_int, _dp, _dp, _dp]
        L.orc_ker2_lanczos.restype = None
        L.orc_subset_solve.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_longlong, _ip, C.c_int,
                                       _dp, _dp, _dp]
        L.orc_subset_solve.restype = C.c_int
        L.orc_batch.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_longlong, _ip, _lp, C.c_longlong,
                                C.c_int, _dp, _dp, _dp, _ip, _dp, _dp, C.c_int]
        L.orc_batch.restype = None
        L.orc_use_impl.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_use_impl.restype = None
        L.orc_splitmix64.argtypes = [C.c_uint64]
        L.orc_splitmix64.restype = C.c_uint64
        L.orc_gen_k.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_int, C.c_int]
        L.orc_gen_k.restype = C.c_int
        L.orc_gen_set.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_int, _ip]
        L.orc_gen_set.restype = None
        L.orc_gen_stream.argtypes = [C.c_uint64, C.c_longlong, C.c_longlong, C.c_int, C.c_int, C.c_int,
                                     C.c_int, _lp, _ip]
        L.orc_gen_stream.restype = C.c_longlong
        L.orc_sturm_count.argtypes = [_dp, _dp, C.c_int, C.c_double]
        L.orc_sturm_count.restype = C.c_int
        L.orc_gershgorin.argtypes = [_dp, _dp, C.c_int, _dp, _dp]
        L.orc_gershgorin.restype = None
        L.orc_bisect_all.argtypes = [_dp, _dp, C.c_int, _dp]
        L.orc_upper_power.restype = C.c_double
        L.orc_upper_power.argtypes = [_dp, C.c_int]
        L.orc_dsg_b.restype = None
        L.orc_dsg_b.argtypes = [_dp, _dp, C.c_int, C.c_int, _ip, C.c_int, C.c_int]
        L.orc_bisect_all.restype = None
        _lib = L
    return _lib


def ref_lib():
    """The reference's own TQLRAT/DET_TRIDIAG (oracle/_ref), or None if not built."""
    global _ref
    if _ref is None and os.path.exists(REF_PATH):
        R = C.CDLL(REF_PATH)
        R.plref_tqlrat.argtypes = [C.c_int, _dp, _dp]
        R.plref_tqlrat.restype = C.c_int
        R.plref_det_tridiag.argtypes = [C.c_int, _dp, _dp]
        R.plref_det_tridiag.restype = C.c_double
        _ref = R
    return _ref


def use_reference_tqlrat(on: bool = True) -> bool:
    """Route the oracle's batch through the reference's compiled TQLRAT."""
    R = ref_lib() if on else None
    if R is None:
        lib().orc_use_impl(None, None)
        return False
    lib().orc_use_impl(C.cast(R.plref_tqlrat, C.c_void_p), C.cast(R.plref_det_tridiag, C.c_void_p))
    return True


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _l(a):
    return a.ctypes.data_as(_lp)


# ----------------------------------------------------------------------------- tridiagonal


def tqlrat(d, e2, impl: str = "oracle"):
    """EISPACK TQLRAT on copies of (d, e2); returns (eigs ascending, e2_after, ierr)."""
    d = np.array(d, dtype=np.float64)
    e2 = np.array(e2, dtype=np.float64)
    f = ref_lib().plref_tqlrat if impl == "reference" else lib().orc_tqlrat
    ierr = f(len(d), _d(d), _d(e2))
    return d, e2, ierr


def det_tridiag(a, b, impl: str = "oracle") -> float:
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    f = ref_lib().plref_det_tridiag if impl == "reference" else lib().orc_det_tridiag
    return float(f(len(a), _d(a), _d(b)))


def ker2_lanczos(As):
    """FP64 KER2 recurrence on a k x k matrix: (alpha[k], beta[k+2])."""
    As = np.ascontiguousarray(As, dtype=np.float64)
    k = As.shape[0]
    alpha = np.zeros(k + 2)
    beta = np.zeros(k + 2)
    work = np.zeros(4 * k)
    lib().orc_ker2_lanczos(_d(As), k, _d(alpha), _d(beta), _d(work))
    return alpha[:k].copy(), beta


def subset_solve(A, S):
    """One set through the reference path restated: (eigs ascending, det, ierr)."""
    A = np.ascontiguousarray(A)
    isd = 1 if A.dtype == np.float64 else 0
    if not isd:
        A = np.ascontiguousarray(A, dtype=np.float32)
    S = np.ascontiguousarray(S, dtype=np.int32)
    k = len(S)
    eig = np.zeros(k)
    det = np.zeros(1)
    work = np.zeros(k * k + 8 * k + 8)
    ierr = lib().orc_subset_solve(A.ctypes.data, isd, A.shape[0], A.shape[1], _i(S), k, _d(eig),
                                  _d(det), _d(work))
    return eig, float(det[0]), int(ierr)


def batch(A, idx, k=None, offsets=None, want_all=False, want_det=False, nthreads=0):
    """OpenMP batch over sets.  Returns dict(lmin, lmax, delta, err[, eig][, det])."""
    A = np.ascontiguousarray(A)
    isd = 1 if A.dtype == np.float64 else 0
    if not isd:
        A = np.ascontiguousarray(A, dtype=np.float32)
    idx = np.ascontiguousarray(idx, dtype=np.int32).reshape(-1)
    if offsets is not None:
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        nsets = len(offsets) - 1
        kk = 0
    else:
        nsets = len(idx) // k
        kk = k
    out = dict(lmin=np.zeros(nsets), lmax=np.zeros(nsets), delta=np.zeros(nsets),
               err=np.zeros(nsets, dtype=np.int32))
    eig = np.zeros(len(idx)) if want_all else None
    det = np.zeros(nsets) if want_det else None
    lib().orc_batch(A.ctypes.data, isd, A.shape[0], A.shape[1], _i(idx),
                    _l(offsets) if offsets is not None else None, nsets, kk,
                    _d(out["lmin"]), _d(out["lmax"]), _d(out["delta"]), _i(out["err"]),
                    _d(eig) if eig is not None else None, _d(det) if det is not None else None,
                    int(nthreads))
    if eig is not None:
        out["eig"] = eig
    if det is not None:
        out["det"] = det
    return out


# ----------------------------------------------------------------------------- generator


def gen_set(seed: int, s: int, n: int, k: int):
    out = np.zeros(k, dtype=np.int32)
    lib().orc_gen_set(seed, s, n, k, _i(out))
    return out


def gen_k(seed: int, s: int, kdist: int, kmin: int, kmax: int) -> int:
    return int(lib().orc_gen_k(seed, s, kdist, kmin, kmax))


def gen_stream(seed: int, first: int, nsets: int, n: int, kdist: int = 0, kmin: int = 16, kmax: int = 16):
    """(offsets int64[nsets+1], idx int32[total]) for sets first..first+nsets-1."""
    total = lib().orc_gen_stream(seed, first, nsets, n, kdist, kmin, kmax, None, None)
    offsets = np.zeros(nsets + 1, dtype=np.int64)
    idx = np.zeros(total, dtype=np.int32)
    lib().orc_gen_stream(seed, first, nsets, n, kdist, kmin, kmax, _l(offsets), _i(idx))
    return offsets, idx


# ----------------------------------------------------------------------------- Sturm


def sturm_count(alpha, beta2, x: float) -> int:
    alpha = np.ascontiguousarray(alpha, dtype=np.float64)
    beta2 = np.ascontiguousarray(beta2, dtype=np.float64)
    return int(lib().orc_sturm_count(_d(alpha), _d(beta2), len(alpha), float(x)))


def bisect_all(alpha, beta2):
    alpha = np.ascontiguousarray(alpha, dtype=np.float64)
    beta2 = np.ascontiguousarray(beta2, dtype=np.float64)
    eig = np.zeros(len(alpha))
    lib().orc_bisect_all(_d(alpha), _d(beta2), len(alpha), _d(eig))
    return eig


def dsg_b(frame, subset, off: int = 0):
    """FP64 Gram block of frame columns `subset` (DSG_B, ParaLanczos.cu:364-382)."""
    frame = np.ascontiguousarray(frame, dtype=np.float64)
    subset = np.ascontiguousarray(subset, dtype=np.int32)
    M, N = frame.shape
    n = len(subset)
    out = np.zeros((n, n))
    lib().orc_dsg_b(_d(out), _d(frame), M, N, _i(subset), n, off)
    return out


def upper_power(A) -> float:
    """UPPER_KER's ||A||_2 estimate (ParaLanczos.cu:1484-1626), all-ones start."""
    A = np.ascontiguousarray(A, dtype=np.float64)
    return lib().orc_upper_power(_d(A), A.shape[0])


# ----------------------------------------------------------------------------- LAPACK truth


def dsyev_eigs(As):
    """FP64 LAPACK dsyev eigenvalues (ascending) of a symmetric matrix."""
    from scipy.linalg import lapack
    w, _, info = lapack.dsyev(np.asarray(As, dtype=np.float64), compute_v=0)
    if info != 0:
        raise RuntimeError(f"dsyev info={info}")
    return w


def dsyev_batch(A, idx, k=None, offsets=None):
    """dsyev truth per set: list of eigenvalue arrays (FP64 submatrix of A)."""
    A64 = np.asarray(A, dtype=np.float64)
    idx = np.asarray(idx).reshape(-1)
    out = []
    if offsets is None:
        n = len(idx) // k
        for s in range(n):
            S = idx[s * k:(s + 1) * k]
            out.append(dsyev_eigs(A64[np.ix_(S, S)]))
    else:
        for s in range(len(offsets) - 1):
            S = idx[offsets[s]:offsets[s + 1]]
            out.append(dsyev_eigs(A64[np.ix_(S, S)]))
    return out
