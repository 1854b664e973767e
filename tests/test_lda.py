"""A matrix with a leading dimension larger than its order (a view of the
first n columns of a wider row-major array): every kernel shape must read
only A[i][j] for i, j < n at i * lda + j.  The padding columns hold NaN, so a
stray read would surface as PL_SET_NONFINITE; the results must be bitwise
those of the same matrix stored densely.
"""
import numpy as np
import pytest

from oracle import oracle as O
from paralanczos_b200 import _lib, api

pytestmark = pytest.mark.gpu


def _padded(A, pad):
    n = A.shape[0]
    P = np.full((n, n + pad), np.nan, dtype=np.float32)
    P[:, :n] = A
    return P


def _solve_view(P, n, idx, k=None, offsets=None):
    """pl_solve on the first n columns of the device copy of P (lda = P's width)."""
    import torch
    Pd = torch.from_numpy(P).cuda()
    view = Pd[:, :n]
    assert view.stride(0) == P.shape[1]
    out = api.solve(view, torch.from_numpy(idx).cuda(), k=k,
                    offsets=None if offsets is None else torch.from_numpy(offsets).cuda())
    torch.cuda.synchronize()
    return {name: t.cpu().numpy() for name, t in out.items()}


def _solve_dense(A, idx, k=None, offsets=None):
    import torch
    out = api.solve(torch.from_numpy(A).cuda(), torch.from_numpy(idx).cuda(), k=k,
                    offsets=None if offsets is None else torch.from_numpy(offsets).cuda())
    torch.cuda.synchronize()
    return {name: t.cpu().numpy() for name, t in out.items()}


def _gram(M, N, seed):
    rng = np.random.default_rng(seed)
    Phi = rng.standard_normal((M, N)) / np.sqrt(M)
    return (Phi.T @ Phi).astype(np.float32)


@pytest.mark.parametrize("k", [8, 16, 32, 48, 64, 96, 128, 192, 256])
def test_uniform_k_with_padded_rows(k):
    n = 1024
    A = _gram(512, n, 20 + k)
    nsets = 2000 if k <= 128 else 150
    _, idx = O.gen_stream(60 + k, 0, nsets, n, 0, k, k)
    for pad in (13, 64):
        r = _solve_view(_padded(A, pad), n, idx, k=k)
        d = _solve_dense(A, idx, k=k)
        assert ((r["err"] & ~_lib.PL_SET_BREAKDOWN) == 0).all()
        for name in ("lmin", "lmax", "delta", "err"):
            np.testing.assert_array_equal(r[name], d[name], err_msg=f"k={k} pad={pad} {name}")


def test_uneven_k_with_padded_rows():
    n = 1024
    A = _gram(512, n, 7)
    offsets, idx = O.gen_stream(61, 0, 3000, n, 2, 1, 256)  # k uniform in [1, 256]
    r = _solve_view(_padded(A, 29), n, idx, offsets=offsets)
    d = _solve_dense(A, idx, offsets=offsets)
    assert ((r["err"] & ~_lib.PL_SET_BREAKDOWN) == 0).all()
    for name in ("lmin", "lmax", "delta", "err"):
        np.testing.assert_array_equal(r[name], d[name], err_msg=name)
