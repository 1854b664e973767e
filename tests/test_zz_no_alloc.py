"""pl_solve_noalloc: the allocation-free entry point for callers that cannot
call cudaMalloc (a host runtime that owns the device-memory budget, code that
runs during a CUDA graph capture, plugins that must not allocate after
start-up).  Its scratch is a static device array inside the library, so this
test checks it against the ordinary entry point, pl_solve, on two calls in a
row (the array keeps the previous call's contents, which must not leak into
the next result).  Kept in a file that sorts last so a stop-at-first-failure
run has already run every other test; it also passes alone in a fresh
process."""
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


def _noalloc(A, idx, k):
    import torch
    nsets = idx.numel() // k
    out = {n: torch.full((nsets,), -7.0, dtype=torch.float64, device="cuda") for n in ("lmin", "lmax", "delta")}
    out["err"] = torch.full((nsets,), -7, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream()
    rc = _lib.lib().pl_solve_noalloc(A.data_ptr(), A.shape[0], A.stride(0), idx.data_ptr(), nsets, k,
                                     out["lmin"].data_ptr(), out["lmax"].data_ptr(),
                                     out["delta"].data_ptr(), out["err"].data_ptr(), st.cuda_stream)
    torch.cuda.synchronize()
    return rc, {n: t.cpu().numpy() for n, t in out.items()}


def test_noalloc_matches_pl_solve_on_two_calls_in_a_row():
    import torch
    for call, (k, nsets, seed) in enumerate([(64, 3000, 11), (16, 5000, 12)]):
        A_np = _gram(1024, 2048, seed)
        _, idx_np = O.gen_stream(seed, 0, nsets, 2048, 0, k, k)
        A = torch.from_numpy(A_np).cuda()
        idx = torch.from_numpy(idx_np).cuda()
        rc, na = _noalloc(A, idx, k)
        assert rc == _lib.PL_OK, f"call {call}: status {rc}"
        ref = {n: t.cpu().numpy() for n, t in api.solve(A, idx, k=k).items()}
        for n in ("lmin", "lmax", "delta"):
            np.testing.assert_allclose(na[n], ref[n], rtol=RTOL, atol=0)
        np.testing.assert_array_equal(na["err"], ref["err"])


def test_noalloc_rejects_k_beyond_its_limit():
    import torch
    A = torch.eye(128, dtype=torch.float32, device="cuda")
    idx = torch.arange(65, dtype=torch.int32, device="cuda")
    rc, _ = _noalloc(A, idx, 65)
    assert rc == _lib.PL_ENOTSUP
