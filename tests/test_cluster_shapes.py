"""Every thread-block-cluster shape of the large-k bins (one or several rows
per thread, one or several CTAs per set) and every symmetric-tile shape (A_S
and P as upper 32 x 32 tiles, one set per CTA), forced as its bin's kernel,
in the extremes mode: random Gram subsets, zero-padded k (including sets
that leave whole tile blocks empty), and breakdown restarts
(a block-diagonal matrix whose all-ones start vector spans an invariant
subspace), against FP64 LAPACK dsyev / numpy eigvalsh within 1e-5 relative.
"""
import numpy as np
import pytest

from oracle import oracle as O
from paralanczos_b200 import _lib, api

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _cluster_variants():
    """(bin, variant) pairs, read from the library's table (host code, no GPU);
    empty if the library is not built, so collection never fails."""
    try:
        return _list_cluster_variants()
    except Exception:
        return []


def _list_cluster_variants():
    out = []
    for b in range(api.num_bins()):
        nvar, _ = api.tune_describe(b, 0)
        for v in range(nvar):
            d = api.tune_describe(b, v)[1]
            if d.startswith("sym") or (d.startswith("cluster") and api.bin_kmax(b) > 128):
                out.append((b, v))
    return out


def _solve(A, idx, k, b, v):
    import torch
    api.tune_set(b, v)
    try:
        out = api.solve(torch.from_numpy(A).cuda(), torch.from_numpy(idx).cuda(), k=k)
        torch.cuda.synchronize()
    finally:
        api.tune_set(b, -1)
    return {n: t.cpu().numpy() for n, t in out.items()}


@pytest.mark.parametrize("bv", _cluster_variants())
def test_cluster_shape(bv):
    b, v = bv
    kmax = api.bin_kmax(b)
    rng = np.random.default_rng(100 + b * 10 + v)
    Phi = rng.standard_normal((1024, 2048)) / np.sqrt(1024)
    A = (Phi.T @ Phi).astype(np.float32)
    for k in (kmax, kmax - 13, kmax - 40):
        _, idx = O.gen_stream(200 + k, 0, 6, 2048, 0, k, k)
        res = _solve(A, idx, k, b, v)
        assert ((res["err"] & ~_lib.PL_SET_BREAKDOWN) == 0).all()
        for s, t in enumerate(O.dsyev_batch(A, idx, k=k)):
            assert abs(res["lmin"][s] - t[0]) <= RTOL * abs(t[0]), (k, s, res["lmin"][s], t[0])
            assert abs(res["lmax"][s] - t[-1]) <= RTOL * abs(t[-1]), (k, s, res["lmax"][s], t[-1])
    k = kmax - 4
    B = (np.kron(np.eye(2), np.ones((k // 2, k // 2))) + np.eye(k)).astype(np.float32)
    res = _solve(B, np.arange(k, dtype=np.int32), k, b, v)
    t = np.linalg.eigvalsh(B.astype(np.float64))
    assert res["err"][0] & _lib.PL_SET_BREAKDOWN
    assert abs(res["lmin"][0] - t[0]) <= RTOL * abs(t[0])
    assert abs(res["lmax"][0] - t[-1]) <= RTOL * abs(t[-1])
