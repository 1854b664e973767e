"""The shared-A engine with two threads per row (k_sa2_solve), forced as the
kernel of the 64 < k <= 96 and 96 < k <= 128 bins, against FP64 LAPACK dsyev: uniform k (full and
zero-padded), uneven k with bad indices, breakdown restarts, NaN input, and
pre-formed Gram blocks (its float4 path).  Extremes only: the all-eigenvalue
mode of the bin uses the other shapes.
"""
import contextlib

import numpy as np
import pytest

from oracle import oracle as O
from paralanczos_b200 import _lib, api

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _bins():
    """The bins this engine serves: 64 < k <= 96 and 96 < k <= 128."""
    return [b for b in range(api.num_bins()) if api.bin_kmax(b) in (96, 128)]


def _variant(b):
    nvar, _ = api.tune_describe(b, 0)
    return next(v for v in range(nvar) if "2 threads/row" in api.tune_describe(b, v)[1])


@contextlib.contextmanager
def _forced():
    bins = _bins()
    assert len(bins) == 2
    for b in bins:
        api.tune_set(b, _variant(b))
    try:
        yield
    finally:
        for b in bins:
            api.tune_set(b, -1)


def _gram(M, N, seed):
    rng = np.random.default_rng(seed)
    Phi = rng.standard_normal((M, N)) / np.sqrt(M)
    return (Phi.T @ Phi).astype(np.float32)


def _run(A, idx, k=None, offsets=None):
    import torch
    with _forced():
        out = api.solve(torch.from_numpy(A).cuda(), torch.from_numpy(idx).cuda(), k=k,
                        offsets=None if offsets is None else torch.from_numpy(offsets).cuda())
        torch.cuda.synchronize()
    return {n: t.cpu().numpy() for n, t in out.items()}


def _check(A, idx, res, k=None, offsets=None, skip=()):
    truth = O.dsyev_batch(A, idx, k=k, offsets=offsets)
    for s, t in enumerate(truth):
        if s in skip:
            continue
        assert abs(res["lmin"][s] - t[0]) <= RTOL * abs(t[0]), (s, res["lmin"][s], t[0])
        assert abs(res["lmax"][s] - t[-1]) <= RTOL * abs(t[-1]), (s, res["lmax"][s], t[-1])
        assert res["delta"][s] == max(1 - res["lmin"][s], res["lmax"][s] - 1)


@pytest.mark.parametrize("k", [128, 97, 96, 65])
def test_uniform_k_vs_dsyev(k):
    A = _gram(1024, 4096, 0)
    _, idx = O.gen_stream(60 + k, 0, 1200, 4096, 0, k, k)
    res = _run(A, idx, k=k)
    assert ((res["err"] & ~_lib.PL_SET_BREAKDOWN) == 0).all()
    _check(A, idx, res, k=k)


def test_uneven_k_with_bad_indices():
    A = _gram(512, 2048, 1)
    rng = np.random.default_rng(7)
    ks = rng.integers(65, 129, size=900)
    offsets = np.zeros(len(ks) + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(ks)
    idx = np.concatenate([rng.choice(2048, size=k, replace=False) for k in ks]).astype(np.int32)
    bad = [0, 450, 899]
    for s in bad:
        idx[offsets[s] + 3] = -1 - s
    res = _run(A, idx, offsets=offsets)
    for s in bad:
        assert res["err"][s] & _lib.PL_SET_BAD_INDEX and np.isnan(res["lmin"][s])
    good = np.setdiff1d(np.arange(len(ks)), bad)
    assert ((res["err"][good] & ~_lib.PL_SET_BREAKDOWN) == 0).all()
    _check(A, idx, res, offsets=offsets, skip=set(bad))


@pytest.mark.parametrize("k", [128, 100, 96, 66])
def test_breakdown_restart_extremes(k):
    for A in (np.eye(k, dtype=np.float32) * 2.0,
              np.kron(np.eye(2), np.ones((k // 2, k // 2))).astype(np.float32) + np.eye(k, dtype=np.float32)):
        res = _run(A, np.arange(k, dtype=np.int32), k=k)
        t = np.linalg.eigvalsh(A.astype(np.float64))
        assert res["err"][0] & _lib.PL_SET_BREAKDOWN
        assert abs(res["lmin"][0] - t[0]) <= RTOL * abs(t[0])
        assert abs(res["lmax"][0] - t[-1]) <= RTOL * abs(t[-1])


def test_nonfinite_input():
    A = _gram(256, 1024, 3)
    A[11, :] = np.nan
    A[:, 11] = np.nan
    _, idx = O.gen_stream(71, 0, 600, 1024, 0, 90, 90)
    res = _run(A, idx, k=90)
    has = (idx.reshape(-1, 90) == 11).any(axis=1)
    assert has.any() and (res["err"][has] & _lib.PL_SET_NONFINITE).all()
    assert ((res["err"][~has] & ~_lib.PL_SET_BREAKDOWN) == 0).all()


@pytest.mark.parametrize("k", [128, 96])
def test_preformed_gram_blocks(k):
    """The on-the-fly Gram form's shape (Phi 2048 x 4096, k = 128; and k = 96)
    solved on its pre-formed blocks: within 1e-5 relative of dsyev on the FP64
    Gram."""
    import torch
    rng = np.random.default_rng(9)
    M, N = 2048, 4096
    Phi = (rng.standard_normal((M, N)) / np.sqrt(M)).astype(np.float32)
    gf = api.GramFrame(torch.from_numpy(Phi).cuda())
    _, idx = O.gen_stream(73, 0, 200, N, 0, k, k)
    di = torch.from_numpy(idx).cuda()
    with _forced():
        out = gf.solve(di, k)
        torch.cuda.synchronize()
    assert ((out["err"].cpu().numpy() & ~_lib.PL_SET_BREAKDOWN) == 0).all()
    lmin, lmax = out["lmin"].cpu().numpy(), out["lmax"].cpu().numpy()
    Phi64 = Phi.astype(np.float64)
    S = idx.reshape(-1, k)
    for s in range(len(S)):
        X = Phi64[:, S[s]]
        w = O.dsyev_eigs(X.T @ X)
        assert abs(lmin[s] - w[0]) <= RTOL * abs(w[0]), (s, lmin[s], w[0])
        assert abs(lmax[s] - w[-1]) <= RTOL * abs(w[-1]), (s, lmax[s], w[-1])
