"""The reference's kernels launched with MATLAB's geometry.

Matlab/gpu_multi_subsvd2.m launches POS_SYM_SUBMATRIX_KER2 on L/128 blocks of
32 threads with subn = minor; gpu_multi_subsvd.m launches POS_SYM_SUBMATRIX_KER
on L/minor blocks of minor/4 threads; gpu_svd.m launches POS_SYM_MAT_KER on one
block of n/4 threads.  MATLAB is not available here, so these tests launch the
library's kernels of the same names through pl_launch_reference_kernel with
those geometries and FP64 device buffers, as CUDAKernel would, and check the
outputs in the reference's layout against LAPACK dsyev (all eigenvalues,
1e-5 of the set's largest) and the oracle (Gram kernels, power iteration).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _launch(name, grid, block, args, block_y=1):
    import torch

    from paralanczos_b200._lib import check, lib
    vals = []
    for a in args:
        if isinstance(a, int):
            vals.append(C.c_int(a))
        else:
            vals.append(C.c_void_p(a.data_ptr()))
    arr = (C.c_void_p * len(vals))(*[C.cast(C.pointer(v), C.c_void_p) for v in vals])
    check(lib().pl_launch_reference_kernel(name.encode(), grid, block, block_y, arr, None),
          "pl_launch_reference_kernel")
    torch.cuda.synchronize()


def _gram(m, n, seed):
    rng = np.random.default_rng(seed)
    Phi = rng.standard_normal((m, n)) / np.sqrt(m)
    return Phi.T @ Phi


def _sets(rng, nsets, n, k):
    return np.stack([rng.choice(n, size=k, replace=False) for _ in range(nsets)]).astype(np.int32)


def _check_all(A, S, eig, det, err):
    from oracle import oracle as O
    k = S.shape[1]
    for s in range(S.shape[0]):
        w = O.dsyev_eigs(A[np.ix_(S[s], S[s])])
        e = eig[s * k:(s + 1) * k]
        assert np.max(np.abs(e - w)) <= 1e-5 * np.max(np.abs(w)), (s, np.max(np.abs(e - w)))
        assert abs(det[s] - np.prod(w)) <= 1e-4 * abs(np.prod(w))
        assert err[s] == 0


@pytest.mark.parametrize("subn", [4, 8, 16, 32, 64, 128])
def test_ker2_matlab_geometry(subn):
    import torch
    rng = np.random.default_rng(subn)
    n = 600
    A = _gram(300, n, 1)
    nsets = max(1, 256 // subn) * 3
    L = nsets * subn
    assert L % 128 == 0
    S = _sets(rng, nsets, n, subn)
    dA = torch.from_numpy(A).cuda()
    dS = torch.from_numpy(S.reshape(-1)).cuda()
    eig = torch.full((L,), -7.0, dtype=torch.float64, device="cuda")
    det = torch.zeros(nsets, dtype=torch.float64, device="cuda")
    err = torch.full((nsets,), -1, dtype=torch.int32, device="cuda")
    _launch("POS_SYM_SUBMATRIX_KER2", L // 128, 32, [dA, n, det, eig, err, dS, subn])
    _check_all(A, S, eig.cpu().numpy(), det.cpu().numpy(), err.cpu().numpy())


@pytest.mark.parametrize("subn", [4, 12, 48, 128])
def test_ker_matlab_geometry(subn):
    import torch
    rng = np.random.default_rng(100 + subn)
    n = 500
    A = _gram(400, n, 2)
    nsets = 37
    S = _sets(rng, nsets, n, subn)
    dA = torch.from_numpy(A).cuda()
    dS = torch.from_numpy(S.reshape(-1)).cuda()
    eig = torch.zeros(nsets * subn, dtype=torch.float64, device="cuda")
    det = torch.zeros(nsets, dtype=torch.float64, device="cuda")
    err = torch.full((nsets,), -1, dtype=torch.int32, device="cuda")
    _launch("POS_SYM_SUBMATRIX_KER", nsets, subn // 4, [dA, n, det, eig, err, dS, subn])
    _check_all(A, S, eig.cpu().numpy(), det.cpu().numpy(), err.cpu().numpy())


def test_mat_kernel_and_example_matrix():
    """POS_SYM_MAT_KER on the reference's own 8x8 example (example1.cu:19-26)
    and on a 96x96 Gram matrix."""
    import json
    import os

    import torch
    fx = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "fixture8.json")))
    ex = np.asarray(fx["matrix"], dtype=np.float64)
    ex = ex.reshape(int(round(np.sqrt(ex.size))), -1)
    for A in (ex, _gram(200, 96, 3)):
        n = A.shape[0]
        dA = torch.from_numpy(np.ascontiguousarray(A)).cuda()
        eig = torch.zeros(n, dtype=torch.float64, device="cuda")
        det = torch.zeros(1, dtype=torch.float64, device="cuda")
        err = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        _launch("POS_SYM_MAT_KER", 1, n // 4, [dA, n, det, eig, err])
        _check_all(A, np.arange(n, dtype=np.int32)[None, :], eig.cpu().numpy(), det.cpu().numpy(),
                   err.cpu().numpy())


def test_bad_index_reported_per_set():
    import torch
    n, subn, nsets = 200, 16, 8
    A = _gram(100, n, 4)
    S = _sets(np.random.default_rng(5), nsets, n, subn)
    S[3, 7] = n + 5
    dA = torch.from_numpy(A).cuda()
    dS = torch.from_numpy(S.reshape(-1)).cuda()
    eig = torch.zeros(nsets * subn, dtype=torch.float64, device="cuda")
    det = torch.zeros(nsets, dtype=torch.float64, device="cuda")
    err = torch.full((nsets,), -1, dtype=torch.int32, device="cuda")
    _launch("POS_SYM_SUBMATRIX_KER2", nsets * subn // 128, 32, [dA, n, det, eig, err, dS, subn])
    e = err.cpu().numpy()
    assert e[3] == 4 and np.isnan(eig.cpu().numpy()[3 * subn:4 * subn]).all()
    assert (e[[0, 1, 2, 4, 5, 6, 7]] == 0).all()


def test_upper_kernel_matches_oracle():
    import torch

    from oracle import oracle as O
    for n in (32, 128, 500):
        A = _gram(2 * n, n, 6)
        dA = torch.from_numpy(A).cuda()
        up = torch.zeros(1, dtype=torch.float64, device="cuda")
        _launch("UPPER_KER", 1, max(1, n // 4), [dA, n, up])
        assert abs(up.item() - O.upper_power(A)) <= 1e-12 * O.upper_power(A)


def test_gram_kernels_match_oracle():
    import torch

    from oracle import oracle as O
    rng = np.random.default_rng(7)
    M, N = 77, 300
    F = rng.standard_normal((M, N))
    dF = torch.from_numpy(F).cuda()
    for n, off in ((16, 0), (32, 3)):
        S = rng.choice(N - off, size=n, replace=False).astype(np.int32)
        dS = torch.from_numpy(S).cuda()
        ref = O.dsg_b(F, S, off=off)
        out = torch.zeros(n * n, dtype=torch.float64, device="cuda")
        _launch("DSG_B", 1, n, [out, dF, M, N, dS, n, off], block_y=n)
        assert np.allclose(out.cpu().numpy().reshape(n, n), ref, rtol=1e-13, atol=1e-12)
        out1 = torch.zeros(n * n, dtype=torch.float64, device="cuda")
        _launch("DSG_B1", 1, n, [out1, dF, M, N, dS, off])
        assert np.allclose(out1.cpu().numpy().reshape(n, n), ref, rtol=1e-13, atol=1e-12)
    # SG_B1: Gram of the first d columns over the first d rows of a card-strided frame
    d, card = 24, 40
    G = rng.standard_normal((d, card))
    out = torch.zeros(d * d, dtype=torch.float64, device="cuda")
    _launch("SG_B1", 1, d, [out, torch.from_numpy(G).cuda(), card])
    ref = O.dsg_b(G, np.arange(d, dtype=np.int32))
    assert np.allclose(out.cpu().numpy().reshape(d, d), ref, rtol=1e-13, atol=1e-12)


def test_unknown_kernel_name_rejected():
    from paralanczos_b200._lib import lib
    arr = (C.c_void_p * 1)()
    assert lib().pl_launch_reference_kernel(b"NOT_A_KERNEL", 1, 1, 1, arr, None) == 1
