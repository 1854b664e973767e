"""Host-side API over the C ABI.

Two layers:
  * the reference's entry points with the same names, argument meaning, output
    layout and error behaviour (ParaLanczos.h:39-47; ParaLanczos.cu:1685-1863):
    ``calculate_subeigs3``, ``calculate_subeigs``, ``calculate_subeigs2``,
    ``calculate_eigs`` take numpy buffers and fill the output buffers in place,
    returning the library status (the reference returns void and prints);
  * the batched solver: ``solve`` on device tensors (asynchronous on a CUDA
    stream), ``solve_host`` on numpy arrays (synchronous, end to end), the
    index generator, tuning and measurement helpers.
All compute runs in libparalanczos_b200.so; this module only moves pointers.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import PL_FORM_BATCHED, PL_FORM_PLAIN, check, lib

FORMS = {"batched": PL_FORM_BATCHED, "plain": PL_FORM_PLAIN}


def _np_ptr(a):
    return None if a is None else a.ctypes.data


def _need(a, dtype, name):
    if not isinstance(a, np.ndarray) or a.dtype != dtype or not a.flags.c_contiguous:
        raise TypeError(f"{name} must be a C-contiguous numpy array of {np.dtype(dtype)}")
    return a


# --------------------------------------------------------------------------- drop-ins


def calculate_subeigs3(mat, subIndexLen, matsize, Eigenvalues, Det, subIndex, subn) -> int:
    """ParaLanczos.cu:1811-1863.  mat: FP64 matsize x matsize; subIndex: int32
    [subIndexLen]; Eigenvalues: FP64 [subIndexLen] (ascending per set); Det: FP64
    [subIndexLen // subn].  Returns the status (0 = ok)."""
    _need(mat, np.float64, "mat")
    _need(Eigenvalues, np.float64, "Eigenvalues")
    _need(Det, np.float64, "Det")
    _need(subIndex, np.int32, "subIndex")
    if Eigenvalues.size < subIndexLen or subIndex.size < subIndexLen or mat.size < matsize * matsize:
        return _lib.PL_EINVAL
    if subn > 0 and Det.size < subIndexLen // subn:
        return _lib.PL_EINVAL
    return lib().pl_calculate_subeigs3(mat.ctypes.data, subIndexLen, matsize, Eigenvalues.ctypes.data,
                                       Det.ctypes.data, subIndex.ctypes.data, subn)


def calculate_subeigs(mat, n, Eigenvalues, Det, subIndex, subn) -> int:
    """ParaLanczos.cu:1725-1765: one set of size subn; Eigenvalues[subn], Det[1]."""
    _need(mat, np.float64, "mat")
    _need(Eigenvalues, np.float64, "Eigenvalues")
    _need(Det, np.float64, "Det")
    _need(subIndex, np.int32, "subIndex")
    if Eigenvalues.size < subn or subIndex.size < subn or mat.size < n * n or Det.size < 1:
        return _lib.PL_EINVAL
    return lib().pl_calculate_subeigs(mat.ctypes.data, n, Eigenvalues.ctypes.data, Det.ctypes.data,
                                      subIndex.ctypes.data, subn)


def calculate_subeigs2(mat, n, matsize, Eigenvalues, Det, subIndex, subn) -> int:
    """ParaLanczos.cu:1768-1808: n indices in sets of subn; Eigenvalues[n], Det[0]."""
    _need(mat, np.float64, "mat")
    _need(Eigenvalues, np.float64, "Eigenvalues")
    _need(Det, np.float64, "Det")
    _need(subIndex, np.int32, "subIndex")
    if Eigenvalues.size < n or subIndex.size < n or mat.size < matsize * matsize or Det.size < 1:
        return _lib.PL_EINVAL
    return lib().pl_calculate_subeigs2(mat.ctypes.data, n, matsize, Eigenvalues.ctypes.data,
                                       Det.ctypes.data, subIndex.ctypes.data, subn)


def calculate_eigs(mat, n, Eigenvalues, Det) -> int:
    """ParaLanczos.cu:1685-1722: all eigenvalues of the n x n matrix."""
    _need(mat, np.float64, "mat")
    _need(Eigenvalues, np.float64, "Eigenvalues")
    _need(Det, np.float64, "Det")
    if Eigenvalues.size < n or mat.size < n * n or Det.size < 1:
        return _lib.PL_EINVAL
    return lib().pl_calculate_eigs(mat.ctypes.data, n, Eigenvalues.ctypes.data, Det.ctypes.data)


# --------------------------------------------------------------------------- batched


def solve(A, idx, k=None, offsets=None, form="batched", want_all=False, stream=None, out=None):
    """Solve every set on the GPU.  A: (n, n) float32 CUDA tensor (symmetric);
    idx: int32 CUDA tensor; uniform k, or CSR offsets (int64 CUDA tensor).
    Returns a dict of CUDA tensors lmin, lmax, delta (float64), err (int32) and,
    with want_all, eig (float64, like idx) and det.  Asynchronous on `stream`
    (default: torch's current stream)."""
    import torch
    if A.dtype != torch.float32 or not A.is_cuda or A.dim() != 2:
        raise TypeError("A must be a 2-D float32 CUDA tensor")
    if A.stride(1) != 1:
        raise TypeError("A must be row-major (stride(1) == 1)")
    if idx.dtype != torch.int32 or not idx.is_cuda or not idx.is_contiguous():
        raise TypeError("idx must be a contiguous int32 CUDA tensor")
    if offsets is not None:
        if offsets.dtype != torch.int64 or not offsets.is_cuda or not offsets.is_contiguous():
            raise TypeError("offsets must be a contiguous int64 CUDA tensor")
        nsets = offsets.numel() - 1
        kk = 0
    else:
        if k is None:
            raise TypeError("k is required without offsets")
        nsets = idx.numel() // int(k)
        kk = int(k)
    dev = A.device
    if out is None:
        out = dict(
            lmin=torch.empty(nsets, dtype=torch.float64, device=dev),
            lmax=torch.empty(nsets, dtype=torch.float64, device=dev),
            delta=torch.empty(nsets, dtype=torch.float64, device=dev),
            err=torch.empty(nsets, dtype=torch.int32, device=dev),
        )
        if want_all:
            out["eig"] = torch.empty(idx.numel(), dtype=torch.float64, device=dev)
            out["det"] = torch.empty(nsets, dtype=torch.float64, device=dev)
    st = stream if stream is not None else torch.cuda.current_stream(dev)
    p = lambda name: out[name].data_ptr() if name in out and out[name] is not None else None
    rc = lib().pl_solve(A.data_ptr(), A.shape[0], A.stride(0), idx.data_ptr(),
                        offsets.data_ptr() if offsets is not None else None, nsets, kk, FORMS[form],
                        p("lmin"), p("lmax"), p("delta"), p("err"), p("eig"), p("det"), st.cuda_stream)
    check(rc, "pl_solve")
    return out


def solve_host(A, idx, k=None, offsets=None, form="batched", want_all=False):
    """End-to-end solve from host numpy buffers (float32 A, int32 idx, int64
    offsets); returns numpy outputs.  Synchronous."""
    A = _need(np.ascontiguousarray(A, dtype=np.float32), np.float32, "A")
    idx = _need(np.ascontiguousarray(idx, dtype=np.int32).reshape(-1), np.int32, "idx")
    if offsets is not None:
        offsets = _need(np.ascontiguousarray(offsets, dtype=np.int64), np.int64, "offsets")
        nsets, kk = len(offsets) - 1, 0
    else:
        nsets, kk = len(idx) // int(k), int(k)
    out = dict(lmin=np.empty(nsets), lmax=np.empty(nsets), delta=np.empty(nsets),
               err=np.empty(nsets, dtype=np.int32))
    if want_all:
        out["eig"] = np.empty(len(idx))
        out["det"] = np.empty(nsets)
    rc = lib().pl_solve_host(A.ctypes.data, A.shape[0], A.shape[1], idx.ctypes.data,
                             _np_ptr(offsets), nsets, kk, FORMS[form], out["lmin"].ctypes.data,
                             out["lmax"].ctypes.data, out["delta"].ctypes.data, out["err"].ctypes.data,
                             _np_ptr(out.get("eig")), _np_ptr(out.get("det")))
    check(rc, "pl_solve_host")
    return out


def gather_blocks(A, idx, k: int, stream=None, out=None):
    """(nsets, k, k) float32 blocks A[S,S] on the device and int32 status bits."""
    import torch
    nsets = idx.numel() // int(k)
    if out is None:
        out = (torch.empty((nsets, k, k), dtype=torch.float32, device=A.device),
               torch.empty(nsets, dtype=torch.int32, device=A.device))
    st = stream if stream is not None else torch.cuda.current_stream(A.device)
    check(lib().pl_gather_blocks(A.data_ptr(), A.shape[0], A.stride(0), idx.data_ptr(), nsets, int(k),
                                 out[0].data_ptr(), out[1].data_ptr(), st.cuda_stream), "pl_gather_blocks")
    return out


def gen_sets(seed: int, first: int, nsets: int, n: int, k: int, device="cuda", stream=None):
    """Uniform-k index sets generated on the device (int32 [nsets*k])."""
    import torch
    idx = torch.empty(nsets * k, dtype=torch.int32, device=device)
    st = stream if stream is not None else torch.cuda.current_stream(idx.device)
    check(lib().pl_gen_sets(seed, first, nsets, n, k, idx.data_ptr(), st.cuda_stream), "pl_gen_sets")
    return idx


def gen_stream_host(seed: int, first: int, nsets: int, n: int, kdist: int = 0, kmin: int = 16,
                    kmax: int = 16):
    """(offsets int64[nsets+1], idx int32[total]) from the library's host generator."""
    L = lib()
    total = L.pl_gen_stream_host(seed, first, nsets, n, kdist, kmin, kmax, None, None)
    offsets = np.empty(nsets + 1, dtype=np.int64)
    idx = np.empty(total, dtype=np.int32)
    L.pl_gen_stream_host(seed, first, nsets, n, kdist, kmin, kmax, offsets.ctypes.data, idx.ctypes.data)
    return offsets, idx


def dropin_cache_stats() -> tuple[int, int]:
    """(hits, misses) of the drop-in entry points' device matrix cache on the
    current device: a hit reused the FP32 matrix already on the GPU, a miss
    uploaded and converted the caller's FP64 matrix."""
    import ctypes
    h, m = ctypes.c_longlong(0), ctypes.c_longlong(0)
    lib().pl_dropin_cache_stats(ctypes.byref(h), ctypes.byref(m))
    return int(h.value), int(m.value)


def fp32_peak(stream=None) -> float:
    """Measured FP32 FMA throughput of the current GPU in TFLOP/s."""
    import torch
    st = stream if stream is not None else torch.cuda.current_stream()
    v = C.c_double(0.0)
    check(lib().pl_fp32_peak(C.byref(v), st.cuda_stream), "pl_fp32_peak")
    return v.value


def gather_peak(stream=None) -> float:
    """Measured rate of uniformly random 4-byte loads from an L2-resident array
    (G elements/s): the ceiling of the A[S,S] gather."""
    import torch
    st = stream if stream is not None else torch.cuda.current_stream()
    v = C.c_double(0.0)
    check(lib().pl_gather_peak(C.byref(v), st.cuda_stream), "pl_gather_peak")
    return v.value


def num_bins() -> int:
    return lib().pl_num_bins()


def bin_kmax(b: int) -> int:
    return lib().pl_bin_kmax(b)


def tune_describe(b: int, variant: int = 0) -> tuple[int, str]:
    buf = C.create_string_buffer(256)
    n = lib().pl_tune_describe(b, variant, buf, 256)
    return n, buf.value.decode()


def tune_get(b: int) -> int:
    """The variant bin b runs now (-1 for an unknown bin)."""
    return lib().pl_tune_get(b)


def tune_set(b: int, variant: int) -> None:
    check(lib().pl_tune_set(b, variant), "pl_tune_set")


def release() -> None:
    check(lib().pl_release(), "pl_release")


# --------------------------------------------------------------------------- on-the-fly Gram


class GramFrame:
    """A frame Phi (m x n, the reference's row-major Frame layout) prepared on
    the device for the on-the-fly Gram form (bf16 hi/lo pieces per column).
    The FP32 frame itself is not kept."""

    def __init__(self, Phi, stream=None):
        import torch
        if Phi.dtype != torch.float32 or not Phi.is_cuda or Phi.dim() != 2 or Phi.stride(1) != 1:
            raise TypeError("Phi must be a row-major 2-D float32 CUDA tensor")
        self.m, self.n = int(Phi.shape[0]), int(Phi.shape[1])
        nbytes = lib().pl_gram_prep_bytes(self.m, self.n)
        self.prep = torch.empty(nbytes, dtype=torch.uint8, device=Phi.device)
        st = stream if stream is not None else torch.cuda.current_stream(Phi.device)
        check(lib().pl_gram_prepare(Phi.data_ptr(), Phi.stride(0), self.m, self.n, self.prep.data_ptr(),
                                    st.cuda_stream), "pl_gram_prepare")

    def blocks(self, idx, k: int, stream=None):
        """(nsets, k, k) float32 Gram blocks Phi_S^T Phi_S and int32 status bits."""
        import torch
        nsets = idx.numel() // int(k)
        out = torch.empty((nsets, k, k), dtype=torch.float32, device=self.prep.device)
        err = torch.empty(nsets, dtype=torch.int32, device=self.prep.device)
        st = stream if stream is not None else torch.cuda.current_stream(self.prep.device)
        check(lib().pl_gram_blocks(self.prep.data_ptr(), self.m, self.n, idx.data_ptr(), nsets, int(k),
                                   out.data_ptr(), err.data_ptr(), st.cuda_stream), "pl_gram_blocks")
        return out, err

    def solve(self, idx, k: int, form="batched", want_all=False, stream=None, out=None):
        """Like ``solve`` with A = Phi^T Phi never materialised (1 <= k <= 128)."""
        import torch
        if idx.dtype != torch.int32 or not idx.is_cuda or not idx.is_contiguous():
            raise TypeError("idx must be a contiguous int32 CUDA tensor")
        nsets = idx.numel() // int(k)
        dev = self.prep.device
        if out is None:
            out = dict(lmin=torch.empty(nsets, dtype=torch.float64, device=dev),
                       lmax=torch.empty(nsets, dtype=torch.float64, device=dev),
                       delta=torch.empty(nsets, dtype=torch.float64, device=dev),
                       err=torch.empty(nsets, dtype=torch.int32, device=dev))
            if want_all:
                out["eig"] = torch.empty(nsets * int(k), dtype=torch.float64, device=dev)
                out["det"] = torch.empty(nsets, dtype=torch.float64, device=dev)
        st = stream if stream is not None else torch.cuda.current_stream(dev)
        p = lambda name: out[name].data_ptr() if name in out and out[name] is not None else None
        check(lib().pl_solve_gram(self.prep.data_ptr(), self.m, self.n, idx.data_ptr(), nsets, int(k),
                                  FORMS[form], p("lmin"), p("lmax"), p("delta"), p("err"), p("eig"),
                                  p("det"), st.cuda_stream), "pl_solve_gram")
        return out


# --------------------------------------------------------------------------- serving

SERVE_STATS = ("completed", "sets", "p50_s", "p99_s", "mean_s", "max_s", "busy_s", "arena_peak",
               "arena_bytes", "waves", "loops_running_max", "queued", "loop_launches", "idle_exits",
               "device_bytes", "loops_running")


class Server:
    """Continuous-batching server over device-resident matrices (pl_serve_*).

    Requests are batched on the GPU by device-resident request loops (one
    CUDA graph each, ``max_waves`` of them, requests spread over them by k);
    all of the server's device memory lies within ``budget_bytes``.
    ``submit`` queues a request and returns its id (raises PLError with status
    PL_EBUSY when the pinned pool is full); ``wait`` returns its results as a
    dict of numpy arrays plus ``latency_s`` (submit to completion)."""

    def __init__(self, budget_bytes: int = 1 << 30, host_pool_bytes: int = 1 << 30, max_waves: int = 4):
        self._h = C.c_void_p()
        self._mats = []   # keep the registered tensors alive
        check(lib().pl_serve_create(int(budget_bytes), int(host_pool_bytes), int(max_waves),
                                    C.byref(self._h)), "pl_serve_create")

    def add_matrix(self, A) -> int:
        import torch
        if A.dtype != torch.float32 or not A.is_cuda or A.dim() != 2 or A.stride(1) != 1:
            raise TypeError("A must be a row-major 2-D float32 CUDA tensor")
        torch.cuda.current_stream(A.device).synchronize()
        mid = C.c_int(-1)
        check(lib().pl_serve_add_matrix(self._h, A.data_ptr(), A.shape[0], A.stride(0), C.byref(mid)),
              "pl_serve_add_matrix")
        self._mats.append(A)
        return mid.value

    def submit(self, matrix_id: int, idx, k: int) -> int:
        idx = _need(np.ascontiguousarray(idx, dtype=np.int32).reshape(-1), np.int32, "idx")
        rid = C.c_longlong(0)
        check(lib().pl_serve_submit(self._h, int(matrix_id), idx.ctypes.data, len(idx) // int(k), int(k),
                                    C.byref(rid)), "pl_serve_submit")
        return rid.value

    def try_submit(self, matrix_id: int, idx, k: int):
        """Like submit, but returns None instead of raising when the pool is full."""
        idx = _need(np.ascontiguousarray(idx, dtype=np.int32).reshape(-1), np.int32, "idx")
        rid = C.c_longlong(0)
        rc = lib().pl_serve_submit(self._h, int(matrix_id), idx.ctypes.data, len(idx) // int(k), int(k),
                                   C.byref(rid))
        if rc == _lib.PL_EBUSY:
            return None
        check(rc, "pl_serve_submit")
        return rid.value

    def wait(self, request_id: int, nsets: int, timeout_s: float = 60.0):
        out = dict(lmin=np.empty(nsets), lmax=np.empty(nsets), delta=np.empty(nsets),
                   err=np.empty(nsets, dtype=np.int32))
        lat = C.c_double(0.0)
        check(lib().pl_serve_wait(self._h, int(request_id), float(timeout_s), out["lmin"].ctypes.data,
                                  out["lmax"].ctypes.data, out["delta"].ctypes.data, out["err"].ctypes.data,
                                  C.byref(lat)), "pl_serve_wait")
        out["latency_s"] = lat.value
        return out

    def stats(self) -> dict:
        buf = (C.c_double * len(SERVE_STATS))()
        check(lib().pl_serve_stats(self._h, buf, len(SERVE_STATS)), "pl_serve_stats")
        return dict(zip(SERVE_STATS, list(buf)))

    def reset_stats(self) -> None:
        check(lib().pl_serve_reset_stats(self._h), "pl_serve_reset_stats")

    def close(self) -> None:
        if self._h:
            check(lib().pl_serve_destroy(self._h), "pl_serve_destroy")
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
