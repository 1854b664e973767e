"""pl_solve_noalloc: the allocation-free entry point for callers that cannot
call cudaMalloc (a host runtime that owns the device-memory budget, code that
runs during a CUDA graph capture, plugins that must not allocate after
start-up).  Its scratch is a static device array inside the library.

Checked here, through the C ABI:
  * on two calls in a row (the array keeps the previous call's contents, which
    must not leak into the next result) it returns exactly what pl_solve, the
    ordinary entry point, returns for the same sets (bit for bit: the same
    kernel runs), and both agree with the oracle and FP64 dsyev within 1e-5;
  * in a fresh process, its first call changes the device's free memory by
    nothing (cudaMemGetInfo before and after; the library's modules are loaded
    eagerly by an earlier non-allocating call, so what the first call could
    allocate is only what it asks for itself);
  * k beyond its limit (64) is refused with PL_ENOTSUP.
Kept in a file that sorts last so a stop-at-first-failure run has already run
every other test; it also passes alone in a fresh process.
"""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from oracle import oracle as O
from paralanczos_b200 import _lib, api

pytestmark = pytest.mark.gpu
RTOL = 1e-5
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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
    for call, (k, nsets, seed) in enumerate([(64, 3000, 11), (16, 5000, 12), (48, 4000, 13)]):
        A_np = _gram(1024, 2048, seed)
        _, idx_np = O.gen_stream(seed, 0, nsets, 2048, 0, k, k)
        A = torch.from_numpy(A_np).cuda()
        idx = torch.from_numpy(idx_np).cuda()
        rc, na = _noalloc(A, idx, k)
        assert rc == _lib.PL_OK, f"call {call}: status {rc}"
        ref = {n: t.cpu().numpy() for n, t in api.solve(A, idx, k=k).items()}
        for n in ("lmin", "lmax", "delta", "err"):
            np.testing.assert_array_equal(na[n], ref[n], err_msg=f"call {call}: {n}")
        assert ((na["err"] & ~_lib.PL_SET_BREAKDOWN) == 0).all()
        orc = O.batch(A_np, idx_np, k=k)
        for n in ("lmin", "lmax"):
            np.testing.assert_allclose(na[n], orc[n], rtol=RTOL, atol=0)
        truth = O.dsyev_batch(A_np, idx_np[:200 * k], k=k)
        for s, t in enumerate(truth):
            assert abs(na["lmin"][s] - t[0]) <= RTOL * abs(t[0])
            assert abs(na["lmax"][s] - t[-1]) <= RTOL * abs(t[-1])


FRESH = textwrap.dedent(r"""
    import ctypes, sys
    import numpy as np
    import torch
    sys.path.insert(0, sys.argv[1])
    from paralanczos_b200 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(5)
    Phi = rng.standard_normal((512, 1024)) / np.sqrt(512)
    A = torch.from_numpy((Phi.T @ Phi).astype(np.float32)).cuda()
    k, nsets = 64, 20000
    idx = torch.from_numpy(np.stack([rng.choice(1024, k, replace=False) for _ in range(nsets)])
                           .astype(np.int32).reshape(-1)).cuda()
    outs = [torch.zeros(nsets, dtype=torch.float64, device="cuda") for _ in range(3)]
    err = torch.zeros(nsets, dtype=torch.int32, device="cuda")
    x64 = torch.ones(16, dtype=torch.float64, device="cuda")
    x32 = torch.zeros(16, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    # a first call into the library that allocates nothing: its CUDA runtime
    # starts and (CUDA_MODULE_LOADING=EAGER) loads every module of the library
    assert L.pl_convert_f64_f32(x64.data_ptr(), x32.data_ptr(), 16, None) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    rc = L.pl_solve_noalloc(A.data_ptr(), 1024, 1024, idx.data_ptr(), nsets, k, outs[0].data_ptr(),
                            outs[1].data_ptr(), outs[2].data_ptr(), err.data_ptr(), None)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert rc == 0, rc
    assert bool((outs[0] > 0).all()) and bool((outs[0] <= outs[1]).all())
    print(f"free before {free0} after {free1}")
    sys.exit(0 if free0 == free1 else 3)
""")


def test_noalloc_first_call_in_a_fresh_process_allocates_nothing():
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    r = subprocess.run([sys.executable, "-c", FRESH, ROOT], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stdout + r.stderr


def test_noalloc_rejects_k_beyond_its_limit():
    import torch
    A = torch.eye(128, dtype=torch.float32, device="cuda")
    idx = torch.arange(65, dtype=torch.int32, device="cuda")
    rc, _ = _noalloc(A, idx, 65)
    assert rc == _lib.PL_ENOTSUP
