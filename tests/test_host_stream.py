"""pl_solve_host with the index array in pinned host memory.

For uniform k whose tuned kernel reads each set's indices one set ahead (the
k <= 64 shape), pl_solve_host lets that kernel read a pinned, device-mapped
index array over the host link while it computes, instead of copying the whole
array before the launch; pageable arrays, other k and the CSR form are copied
first.  Both routes must give bit-identical results, bad indices and
non-finite sets included, and agree with the oracle.
"""
import numpy as np
import pytest

from oracle import oracle as O
from paralanczos_b200 import _lib, api

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _gram(M, N, seed):
    rng = np.random.default_rng(seed)
    Phi = rng.standard_normal((M, N)) / np.sqrt(M)
    return (Phi.T @ Phi).astype(np.float32)


def _pinned_solve(A, idx, k):
    import torch
    nsets = idx.size // k
    idx_p = torch.from_numpy(idx).pin_memory()
    A_p = torch.from_numpy(A).pin_memory()
    out = {n: torch.full((nsets,), -7, dtype=torch.int32 if n == "err" else torch.float64).pin_memory()
           for n in ("lmin", "lmax", "delta", "err")}
    rc = _lib.lib().pl_solve_host(A_p.data_ptr(), A.shape[0], A.shape[1], idx_p.data_ptr(), None, nsets, k, 0,
                                  out["lmin"].data_ptr(), out["lmax"].data_ptr(), out["delta"].data_ptr(),
                                  out["err"].data_ptr(), None, None)
    assert rc == _lib.PL_OK, rc
    return {n: t.numpy().copy() for n, t in out.items()}


@pytest.mark.parametrize("k", [64, 50, 16])
def test_pinned_and_pageable_indices_agree(k):
    n = 2048
    A = _gram(512, n, 3)
    A[77, :] = np.nan  # sets containing index 77 are non-finite
    A[:, 77] = np.nan
    nsets = 30000
    _, idx = O.gen_stream(40 + k, 0, nsets, n, 0, k, k)
    idx = idx.copy()
    bad = [0, 1, 12345, nsets - 1]
    for s in bad:
        idx[s * k + (s % k)] = -3 if s % 2 else n + 5
    pageable = api.solve_host(A, idx, k=k)
    pinned = _pinned_solve(A, idx, k)
    for name in ("lmin", "lmax", "delta", "err"):
        np.testing.assert_array_equal(pinned[name], pageable[name], err_msg=name)
    for s in bad:
        assert pinned["err"][s] & _lib.PL_SET_BAD_INDEX
    sets = idx.reshape(nsets, k)
    nan_sets = (sets == 77).any(axis=1)
    nan_sets[bad] = False
    assert nan_sets.any() and (pinned["err"][nan_sets] & _lib.PL_SET_NONFINITE).all()
    good = np.setdiff1d(np.arange(nsets), np.concatenate([bad, np.nonzero(nan_sets)[0]]))
    assert ((pinned["err"][good] & ~_lib.PL_SET_BREAKDOWN) == 0).all()
    sample = good[::150]
    A_clean = A.copy()
    A_clean[77, :] = 0
    A_clean[:, 77] = 0
    orc = O.batch(A_clean, sets[sample].reshape(-1), k=k)
    np.testing.assert_allclose(pinned["lmin"][sample], orc["lmin"], rtol=RTOL, atol=0)
    np.testing.assert_allclose(pinned["lmax"][sample], orc["lmax"], rtol=RTOL, atol=0)
