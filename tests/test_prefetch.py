"""The shared-A engine's prefetch variants (k <= 32 and k <= 64 bins): the next
set's upper triangle is staged in shared memory with cp.async during the
current set's Lanczos steps and mirrored from there.  The staged elements are
the ones the direct gather loads, so every result must be bitwise equal to the
same shape without the prefetch; checked on a uniform stream, on an uneven
(CSR) stream whose sets change k from one set to the next, with sets carrying
an index outside [0, n) and a set whose k is out of range in between (their
neighbours are prefetched around them), and against FP64 dsyev.  The variants
that also hold some float4 chunks of each row of A_S in registers (AREG) are
compared bitwise with the prefetch shape of the same CTA without them.
"""
import numpy as np
import pytest

from oracle import oracle as O
from paralanczos_b200 import _lib, api

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _variants(b, word):
    nvar, _ = api.tune_describe(b, 0)
    return [v for v in range(nvar) if word in api.tune_describe(b, v)[1]]


def _pairs():
    """(bin, prefetch variant, the same shape without prefetch)."""
    try:
        out = []
        for b in range(api.num_bins()):
            if api.bin_kmax(b) not in (32, 64):
                continue
            descs = [api.tune_describe(b, w)[1] for w in range(api.tune_describe(b, 0)[0])]
            for v in _variants(b, "prefetch"):
                d = descs[v]
                if " AREG=" in d:
                    # chunks of A_S in registers: the same prefetch shape (KB,
                    # RPT, CTA) without them is the reference
                    stem = d.split(" REGS=")[0] + " REGS="
                    base = [w for w, e in enumerate(descs) if e.startswith(stem) and " AREG=" not in e]
                else:
                    d = d.replace("sharedA prefetch ", "sharedA ")
                    base = [w for w, e in enumerate(descs) if e == d]
                out.append((b, v, base[0] if base else -1))
        return out
    except Exception:
        return []


def _run(A, idx, b, v, k=None, offsets=None):
    import torch
    api.tune_set(b, v)
    try:
        At = torch.from_numpy(A).cuda()
        it = torch.from_numpy(idx).cuda()
        ot = torch.from_numpy(offsets).cuda() if offsets is not None else None
        out = api.solve(At, it, k=k, offsets=ot)
        torch.cuda.synchronize()
    finally:
        api.tune_set(b, -1)
    return {n: t.cpu().numpy() for n, t in out.items()}


def _gram(seed, m=512, n=2048):
    rng = np.random.default_rng(seed)
    Phi = rng.standard_normal((m, n)) / np.sqrt(m)
    return (Phi.T @ Phi).astype(np.float32)


@pytest.mark.parametrize("bvb", _pairs())
def test_prefetch_uniform_bitwise(bvb):
    b, v, base = bvb
    kmax = api.bin_kmax(b)
    A = _gram(300 + b)
    _, idx = O.gen_stream(41, 0, 6000, A.shape[0], 0, kmax, kmax)
    r = _run(A, idx, b, v, k=kmax)
    assert ((r["err"] & ~_lib.PL_SET_BREAKDOWN) == 0).all(), np.unique(r["err"], return_counts=True)
    if base >= 0:
        r0 = _run(A, idx, b, base, k=kmax)
        np.testing.assert_array_equal(r["err"], r0["err"])
        np.testing.assert_array_equal(r["lmin"], r0["lmin"])
        np.testing.assert_array_equal(r["lmax"], r0["lmax"])
    sample = np.arange(0, 6000, 97)
    truth = O.dsyev_batch(A, idx.reshape(-1, kmax)[sample].ravel(), k=kmax)
    for s, t in zip(sample, truth):
        assert abs(r["lmin"][s] - t[0]) <= RTOL * abs(t[0])
        assert abs(r["lmax"][s] - t[-1]) <= RTOL * abs(t[-1])


@pytest.mark.parametrize("bvb", _pairs())
def test_prefetch_uneven_with_bad_sets(bvb):
    b, v, base = bvb
    kmax = api.bin_kmax(b)
    kmin = kmax // 2 + 1
    A = _gram(400 + b)
    n = A.shape[0]
    rng = np.random.default_rng(500 + b)
    ks = rng.integers(kmin, kmax + 1, size=3000)
    bad_idx = set(range(5, 3000, 211))   # an index outside [0, n)
    bad_k = set(range(17, 3000, 379))    # k outside this bin's kernel: the binning
    parts, offs = [], [0]
    for s, kk in enumerate(ks):
        if s in bad_k:
            kk = kmax + 1                # lands in the next bin, checked there
        S = rng.choice(n, size=kk, replace=False).astype(np.int32)
        if s in bad_idx:
            S[kk // 2] = n + 7 if s % 2 else -3
        parts.append(S)
        offs.append(offs[-1] + kk)
    idx = np.concatenate(parts)
    offsets = np.array(offs, np.int64)
    r = _run(A, idx, b, v, offsets=offsets)
    for s in range(len(ks)):
        if s in bad_idx:
            assert r["err"][s] & _lib.PL_SET_BAD_INDEX and np.isnan(r["lmin"][s]), s
        else:
            assert (r["err"][s] & ~_lib.PL_SET_BREAKDOWN) == 0, (s, r["err"][s])
    if base >= 0:
        r0 = _run(A, idx, b, base, offsets=offsets)
        good = np.array([s not in bad_idx for s in range(len(ks))])
        np.testing.assert_array_equal(r["lmin"][good], r0["lmin"][good])
        np.testing.assert_array_equal(r["lmax"][good], r0["lmax"][good])
        np.testing.assert_array_equal(r["err"], r0["err"])
    for s in range(0, len(ks), 53):
        if s in bad_idx:
            continue
        t = O.dsyev_eigs(A[np.ix_(parts[s], parts[s])].astype(np.float64))
        assert abs(r["lmin"][s] - t[0]) <= RTOL * abs(t[0])
        assert abs(r["lmax"][s] - t[-1]) <= RTOL * abs(t[-1])
