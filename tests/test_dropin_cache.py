"""The drop-in entry points keep the caller's FP64 matrix on the device.

The reference uploads the whole FP64 matrix on every call
(ParaLanczos.cu:1845-1846).  Here calculate_subeigs3 and friends upload and
convert it once (on the device) and reuse it while the caller passes the same
matrix: same address, order and contents (a content hash of the host matrix
per call, computed while a solve on the cached copy runs; a changed hash
re-uploads and solves again).  Checked through the C ABI: the second call on an unchanged matrix
is a cache hit with bit-identical results, a change of one element is a miss
and is seen in the results, and a second matrix is a miss.
"""
import time

import numpy as np
import pytest

import workloads as W
from oracle import oracle as O
from paralanczos_b200 import api

pytestmark = pytest.mark.gpu


def _call(A64, idx, k):
    nsets = len(idx) // k
    eig = np.full(nsets * k, np.nan)
    det = np.full(nsets, np.nan)
    t0 = time.perf_counter()
    assert api.calculate_subeigs3(A64, len(idx), A64.shape[0], eig, det, idx, k) == 0
    return eig, det, time.perf_counter() - t0


def test_second_call_reuses_the_device_matrix():
    A64 = np.array(W.c2_matrix()[0])          # 4096 x 4096 FP64 (128 MB)
    n, k, nsets = A64.shape[0], 16, 2048
    _, idx = api.gen_stream_host(W.SEED_SETS, 0, nsets, n, 0, k, k)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    h0, m0 = api.dropin_cache_stats()
    e1, d1, t1 = _call(A64, idx, k)
    h1, m1 = api.dropin_cache_stats()
    assert (h1, m1) == (h0, m0 + 1)
    e2, d2, t2 = _call(A64, idx, k)
    h2, m2 = api.dropin_cache_stats()
    assert (h2, m2) == (h1 + 1, m1)
    np.testing.assert_array_equal(e1, e2)
    np.testing.assert_array_equal(d1, d2)
    print(f"calculate_subeigs3, 4096^2 FP64 matrix, {nsets} sets: first call {t1 * 1e3:.1f} ms "
          f"(upload + convert), second {t2 * 1e3:.1f} ms (reused)")
    # results are right: extremes against the oracle
    ref = O.batch(A64, idx, k=k)
    e = e1.reshape(nsets, k)
    assert np.max(np.abs(e[:, 0] - ref["lmin"]) / ref["lmin"]) <= 1e-5
    assert np.max(np.abs(e[:, -1] - ref["lmax"]) / ref["lmax"]) <= 1e-5
    # one changed element (in set 0's submatrix) is a miss and is seen
    S = idx[:k]
    B = A64.copy()
    B[S[0], S[0]] += 0.5
    A64[:] = B                                 # same address, new contents
    e3, _, _ = _call(A64, idx, k)
    h3, m3 = api.dropin_cache_stats()
    assert (h3, m3) == (h2, m2 + 1)
    assert not np.array_equal(e3[:k], e1[:k])
    touched = np.array([S[0] in idx[s * k:(s + 1) * k] for s in range(nsets)])
    np.testing.assert_array_equal(e3.reshape(nsets, k)[~touched], e1.reshape(nsets, k)[~touched])
    t = O.dsyev_eigs(B[np.ix_(S, S)])
    assert np.max(np.abs(e3[:k] - t) / np.abs(t)) <= 1e-5


def test_another_matrix_is_a_miss():
    A64, _ = W.c1_matrix()
    A64 = np.array(A64)
    k, nsets = 16, 64
    _, idx = api.gen_stream_host(W.SEED_SETS, 0, nsets, A64.shape[0], 0, k, k)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    _call(A64, idx, k)
    h0, m0 = api.dropin_cache_stats()
    C = A64 * 2.0
    eC, _, _ = _call(C, idx, k)
    h1, m1 = api.dropin_cache_stats()
    assert m1 == m0 + 1 and h1 == h0
    eA, _, _ = _call(A64, idx, k)
    np.testing.assert_allclose(eC, 2.0 * eA, rtol=1e-5)
