"""Parity on the benchmark configurations themselves (the same seeded matrices
and set streams as bench.py; workloads.py builds them), through the C ABI.

  C1  Phi 128 x 512 N(0, 1/128) seed 0; all 10,000 sets of k = 16 (seed 1)
      through the reference's own entry point calculate_subeigs3 (FP64 host
      matrix, all eigenvalues ascending + determinant, ParaLanczos.cu:1811-1863,
      output layout ParaLanczos.cu:1474-1478): every eigenvalue of every set
      against FP64 LAPACK dsyev, the extremes against the oracle.
  C2  Phi 1024 x 4096 N(0, 1/1024) seed 0; the full 1,000,000 sets of k = 64 in
      one batched launch and one plain launch: 2,000 sets (every 500th) against
      the oracle and dsyev in both forms, and size-independent properties on
      all 1,000,000 (status, ordering, delta_k, agreement of the two forms).
  C3  the same A; the 300,000-set stream with k in {8, ..., 256}, P ~ 1/k, in
      one binned launch: at least 200 sets per k against dsyev, 50 per k
      against the oracle; per-k max and p99 printed.

Bar: relative error <= 1e-5 against dsyev and the oracle (lambda_min,
lambda_max; every eigenvalue in the drop-in mode), exact index handling.
"""
import numpy as np
import pytest

import workloads as W
from oracle import oracle as O
from paralanczos_b200 import _lib, api

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _ok(err):
    return ((np.asarray(err) & ~_lib.PL_SET_BREAKDOWN) == 0).all()


def _rel(x, t):
    return np.abs(np.asarray(x) - np.asarray(t)) / np.abs(np.asarray(t))


def _dsyev_extremes(A, idx, offs, sets):
    lo = np.empty(len(sets))
    hi = np.empty(len(sets))
    for j, s in enumerate(sets):
        S = idx[offs[s]:offs[s + 1]]
        w = O.dsyev_eigs(np.asarray(A, dtype=np.float64)[np.ix_(S, S)])
        lo[j], hi[j] = w[0], w[-1]
    return lo, hi


def test_c1_all_sets_through_calculate_subeigs3():
    A64, A32 = W.c1_matrix()
    A64 = np.ascontiguousarray(A64)
    n, k, nsets = W.C1["n"], W.C1["k"], W.C1["nsets"]
    offs, idx = api.gen_stream_host(W.SEED_SETS, 0, nsets, n, 0, k, k)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    eig = np.full(nsets * k, np.nan)
    det = np.full(nsets, np.nan)
    assert api.calculate_subeigs3(A64, nsets * k, n, eig, det, idx, k) == 0
    worst = 0.0
    for s in range(nsets):
        S = idx[s * k:(s + 1) * k]
        t = O.dsyev_eigs(A64[np.ix_(S, S)])
        e = eig[s * k:(s + 1) * k]
        r = np.max(_rel(e, t))
        worst = max(worst, r)
        assert r <= RTOL, (s, r)
        assert np.all(np.diff(e) >= 0)
        assert abs(det[s] - np.prod(t)) <= 1e-4 * abs(np.prod(t))
    # extremes against the oracle (the reference's recurrence restated, FP64)
    ref = O.batch(A64, idx, k=k)
    e2 = eig.reshape(nsets, k)
    assert np.max(_rel(e2[:, 0], ref["lmin"])) <= RTOL
    assert np.max(_rel(e2[:, -1], ref["lmax"])) <= RTOL
    print(f"C1: {nsets} sets, every eigenvalue within {worst:.2e} of dsyev")


@pytest.fixture(scope="module")
def c2_dev():
    import torch
    A32 = np.array(W.c2_matrix()[1])
    A = torch.from_numpy(A32).cuda()
    idx = api.gen_sets(W.SEED_SETS, 0, W.C2["nsets"], W.C2["n"], W.C2["k"])
    return A32, A, idx


def test_c2_full_launch_both_forms(c2_dev):
    import torch
    A32, A, idx = c2_dev
    k, nsets = W.C2["k"], W.C2["nsets"]
    res = {}
    for form in ("batched", "plain"):
        out = api.solve(A, idx, k=k, form=form)
        torch.cuda.synchronize()
        res[form] = {n: t.cpu().numpy() for n, t in out.items()}
    b, p = res["batched"], res["plain"]
    # properties of every one of the 1,000,000 sets
    for r in (b, p):
        assert _ok(r["err"])
        assert np.all(r["lmin"] <= r["lmax"])
        assert np.all(r["lmin"] > 0)
        np.testing.assert_array_equal(r["delta"], np.maximum(1 - r["lmin"], r["lmax"] - 1))
    assert np.max(_rel(b["lmin"], p["lmin"])) <= 2 * RTOL
    assert np.max(_rel(b["lmax"], p["lmax"])) <= 2 * RTOL
    # 2,000 sets against dsyev and the oracle
    sel = np.arange(0, nsets, 500)
    idx_h = idx.view(nsets, k)[torch.from_numpy(sel).cuda()].cpu().numpy()
    sub = np.ascontiguousarray(idx_h.reshape(-1))
    offs = np.arange(0, (len(sel) + 1) * k, k)
    lo, hi = _dsyev_extremes(A32, sub, offs, range(len(sel)))
    ref = O.batch(A32, sub, k=k)
    for form, r in res.items():
        e = np.maximum(_rel(r["lmin"][sel], lo), _rel(r["lmax"][sel], hi))
        eo = np.maximum(_rel(r["lmin"][sel], ref["lmin"]), _rel(r["lmax"][sel], ref["lmax"]))
        print(f"C2 {form}: 2,000 sets, vs dsyev max {e.max():.2e} p99 {np.percentile(e, 99):.2e}; "
              f"vs oracle max {eo.max():.2e}")
        assert e.max() <= RTOL and eo.max() <= RTOL


def test_c3_per_k_vs_dsyev_and_oracle(c2_dev):
    import torch
    A32, A, _ = c2_dev
    n, nsets = W.C3["n"], W.C3["nsets"]
    offs, idx = api.gen_stream_host(W.SEED_SETS, 0, nsets, n, kdist=1)
    ks = np.diff(offs)
    out = api.solve(A, torch.from_numpy(idx).cuda(), offsets=torch.from_numpy(offs).cuda())
    torch.cuda.synchronize()
    r = {nm: t.cpu().numpy() for nm, t in out.items()}
    assert _ok(r["err"])
    assert np.all(r["lmin"] <= r["lmax"])
    for kv in W.C3["kvalues"]:
        sets = np.nonzero(ks == kv)[0]
        assert len(sets) >= 200, (kv, len(sets))
        chk = sets[np.linspace(0, len(sets) - 1, 200).astype(int)]
        lo, hi = _dsyev_extremes(A32, idx, offs, chk)
        e = np.maximum(_rel(r["lmin"][chk], lo), _rel(r["lmax"][chk], hi))
        och = chk[:50]
        sub = np.concatenate([idx[offs[s]:offs[s + 1]] for s in och])
        ref = O.batch(A32, sub, k=kv)
        eo = np.maximum(_rel(r["lmin"][och], ref["lmin"]), _rel(r["lmax"][och], ref["lmax"]))
        print(f"C3 k={kv}: {len(sets)} sets; 200 vs dsyev max {e.max():.2e} p99 {np.percentile(e, 99):.2e}; "
              f"50 vs oracle max {eo.max():.2e}")
        assert e.max() <= RTOL and eo.max() <= RTOL


@pytest.mark.parametrize("kind", ["gauss", "rademacher"])
def test_c4_on_the_fly_gram_2000_sets(kind):
    """C4: Phi 2048 x 16384 (seed 0, Gaussian or Rademacher), A never formed:
    each A[S,S] = Phi_S^T Phi_S on the tensor cores (bf16 split products,
    FP32 accumulation), then the Lanczos.  2,000 of the sets of k = 128 (the
    first 2,000 of the generator's stream) against FP64 dsyev of the FP64 Gram
    of the same FP32 frame columns; max and p99 printed."""
    import torch
    Phi = W.c4_frame(kind)
    k, nsets = W.C4["k"], 2000
    gf = api.GramFrame(torch.from_numpy(Phi).cuda())
    idx = api.gen_sets(W.SEED_SETS, 0, nsets, W.C4["n"], k)
    out = gf.solve(idx, k)
    torch.cuda.synchronize()
    r = {nm: t.cpu().numpy() for nm, t in out.items()}
    assert _ok(r["err"])
    S = idx.view(nsets, k).cpu().numpy()
    errs = np.empty(nsets)
    for s in range(nsets):
        X = Phi[:, S[s]].astype(np.float64)
        w = O.dsyev_eigs(X.T @ X)
        errs[s] = max(abs(r["lmin"][s] - w[0]) / abs(w[0]), abs(r["lmax"][s] - w[-1]) / abs(w[-1]))
    print(f"C4 {kind}: 2,000 sets k=128, vs dsyev max {errs.max():.2e} p99 {np.percentile(errs, 99):.2e}")
    assert errs.max() <= RTOL
