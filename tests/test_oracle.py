"""The CPU oracle, pinned against the reference's own code and LAPACK.

* TQLRAT / DET_TRIDIAG restated in oracle/pl_oracle.c are bit-identical to the
  reference's own routines (ParaLanczos.cu:32-189, 243-269) compiled from its
  source: live against oracle/_ref when built, and against the frozen outputs
  in tests/golden/tqlrat_ref.npz everywhere.
* The restated KER2 path (ParaLanczos.cu:1285-1374 + 1454-1478) reproduces
  LAPACK dsyev on the reference's own 8x8 fixture (example1.cu:19-26).
* The Sturm-count bisection restatement matches dsyev on random tridiagonals.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _tql_cases():
    z = np.load(os.path.join(GOLD, "tqlrat_ref.npz"))
    off = 0
    for i, n in enumerate(z["lens"]):
        sl = slice(off, off + n)
        yield (z["d"][sl], z["e2"][sl], z["out_d"][sl], z["out_e2"][sl], int(z["ierr"][i]),
               float(z["det"][i]))
        off += n


def test_tqlrat_matches_frozen_reference_outputs_bitwise():
    n = 0
    for d, e2, od, oe2, ierr, det in _tql_cases():
        dd, ee, ie = O.tqlrat(d, e2)
        assert ie == ierr
        assert np.array_equal(dd, od)
        assert np.array_equal(ee, oe2)
        dt = O.det_tridiag(dd, ee)
        assert dt == det or (np.isnan(dt) and np.isnan(det))
        n += 1
    assert n >= 30


@pytest.mark.skipif(O.ref_lib() is None, reason="oracle/_ref not built (no reference tree)")
def test_tqlrat_matches_compiled_reference_live():
    rng = np.random.default_rng(5)
    for _ in range(500):
        n = int(rng.integers(1, 100))
        d = rng.standard_normal(n) * 10.0 ** rng.integers(-4, 5)
        e2 = (rng.standard_normal(n) * 10.0 ** rng.integers(-4, 5)) ** 2
        if rng.random() < 0.2:
            e2[rng.integers(0, n)] = 0.0
        a = O.tqlrat(d, e2)
        b = O.tqlrat(d, e2, impl="reference")
        assert a[2] == b[2]
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        da, db = O.det_tridiag(a[0], a[1]), O.det_tridiag(b[0], b[1], impl="reference")
        assert da == db or (np.isnan(da) and np.isnan(db))


def test_tqlrat_eigenvalues_vs_numpy():
    rng = np.random.default_rng(11)
    for n in (2, 5, 16, 40):
        d = rng.standard_normal(n)
        b = rng.standard_normal(n - 1)
        T = np.diag(d) + np.diag(b, 1) + np.diag(b, -1)
        e2 = np.r_[0.0, b * b]
        dd, _, ie = O.tqlrat(d, e2)
        assert ie == 0
        np.testing.assert_allclose(dd, np.linalg.eigvalsh(T), rtol=0, atol=1e-12)


def test_fixture8_oracle_vs_dsyev():
    fx = json.load(open(os.path.join(GOLD, "fixture8.json")))
    g = np.array(fx["matrix"]).reshape(8, 8)
    for c in fx["cases"]:
        S = c["subset"]
        eig, det, ierr = O.subset_solve(g, S)
        truth = O.dsyev_eigs(g[np.ix_(S, S)])
        assert ierr == 0
        np.testing.assert_array_equal(eig, np.array(c["oracle_eigs"]))   # frozen
        np.testing.assert_allclose(eig, truth, rtol=1e-12)              # LAPACK
        np.testing.assert_allclose(det, np.prod(truth), rtol=1e-12)


def test_fixture8_known_values():
    # subset {1,3,5,7} of the reference's example matrix (example1.cu:39-42)
    fx = json.load(open(os.path.join(GOLD, "fixture8.json")))
    g = np.array(fx["matrix"]).reshape(8, 8)
    eig, det, _ = O.subset_solve(g, [1, 3, 5, 7])
    np.testing.assert_allclose(eig, [0.51306705, 2.73205152, 7.03431746, 33.22446398], rtol=1e-7)
    np.testing.assert_allclose(det, 327.59929009, rtol=1e-9)


def test_oracle_sets_frozen_and_vs_dsyev():
    z = np.load(os.path.join(GOLD, "oracle_sets.npz"))
    tags = sorted({k[:-len("_sub")] for k in z.files if k.endswith("_sub")})
    assert tags
    for tag in tags:
        sub = z[tag + "_sub"]
        k = sub.shape[1]
        for s in range(sub.shape[0]):
            eig, det, ierr = O.subset_solve(sub[s], np.arange(k, dtype=np.int32))
            assert ierr == int(z[tag + "_oracle_ierr"][s])
            np.testing.assert_array_equal(eig, z[tag + "_oracle_eig"][s])
            tr = z[tag + "_dsyev_eig"][s]
            # the reference recurrence has no reorthogonalisation: its extremes
            # are accurate, its interior values drift at larger k
            assert abs(eig[0] - tr[0]) / tr[0] < 1e-9
            assert abs(eig[-1] - tr[-1]) / tr[-1] < 1e-9


def test_batch_matches_single():
    rng = np.random.default_rng(3)
    Phi = rng.standard_normal((64, 200)) / 8.0
    A = (Phi.T @ Phi).astype(np.float32)
    offs, idx = O.gen_stream(9, 0, 20, 200, 1, 8, 256)
    idx = idx % 200
    # build valid sets of mixed k <= 64
    sets = [rng.choice(200, size=int(k), replace=False) for k in rng.integers(2, 64, 20)]
    offs = np.r_[0, np.cumsum([len(s) for s in sets])].astype(np.int64)
    flat = np.concatenate(sets).astype(np.int32)
    res = O.batch(A, flat, offsets=offs, want_all=True, want_det=True, nthreads=4)
    for s, S in enumerate(sets):
        eig, det, ierr = O.subset_solve(A, S)
        np.testing.assert_array_equal(res["eig"][offs[s]:offs[s + 1]], eig)
        assert res["lmin"][s] == eig[0] and res["lmax"][s] == eig[-1]
        assert res["delta"][s] == max(1 - eig[0], eig[-1] - 1)


def test_bad_index_reported():
    A = np.eye(4, dtype=np.float32)
    res = O.batch(A, np.array([0, 1, 2, 7], dtype=np.int32), k=4)
    assert res["err"][0] == -1 and np.isnan(res["lmin"][0])


def test_sturm_count_and_bisection():
    rng = np.random.default_rng(17)
    for n in (1, 2, 7, 33, 128, 300):
        a = rng.standard_normal(n) * 3
        b = rng.standard_normal(n) if n > 1 else np.zeros(1)
        b2 = np.r_[0.0, (b[1:] if n > 1 else [])] ** 2 if n > 1 else np.zeros(1)
        T = np.diag(a)
        if n > 1:
            T += np.diag(np.sqrt(b2[1:]), 1) + np.diag(np.sqrt(b2[1:]), -1)
        ev = np.linalg.eigvalsh(T)
        for x in np.r_[ev - 1e-7, ev + 1e-7, rng.standard_normal(5) * 4]:
            assert O.sturm_count(a, b2, x) == int(np.sum(ev < x))
        np.testing.assert_allclose(O.bisect_all(a, b2), ev, rtol=0, atol=1e-12 * max(1, abs(ev).max()))


def test_sturm_decoupled_and_degenerate():
    a = np.array([2.0, 2.0, 2.0, 5.0, 5.0])
    b2 = np.array([0.0, 0.0, 0.0, 0.0, 0.0])
    np.testing.assert_allclose(O.bisect_all(a, b2), np.sort(a), atol=1e-13)
    # minors of 100 rows of 1e20 overflow FP64 without the power-of-two
    # rescaling; the bisection tolerance is relative to the spectrum's scale
    a = np.r_[np.full(100, 1e20), np.full(100, 3.0)]
    b2 = np.r_[0.0, np.full(199, 1.0)]
    T = np.diag(a) + np.diag(np.ones(199), 1) + np.diag(np.ones(199), -1)
    ev = np.linalg.eigvalsh(T)
    np.testing.assert_allclose(O.bisect_all(a, b2), ev, rtol=0, atol=1e-13 * 1e20)
    assert O.sturm_count(a, b2, 1e19) == 100


def test_dsg_b_matches_blas_and_offset():
    """DSG_B restatement (ParaLanczos.cu:364-382): Gram of frame columns S,
    frame row-major M x N, column offset applied to every index."""
    rng = np.random.default_rng(0)
    F = rng.standard_normal((37, 50))
    S = np.array([3, 7, 1, 49], dtype=np.int32)
    G = O.dsg_b(F, S)
    assert np.allclose(G, F[:, S].T @ F[:, S], rtol=0, atol=1e-12)
    assert np.array_equal(G, G.T)
    G1 = O.dsg_b(F, S[:3], off=1)
    assert np.allclose(G1, F[:, S[:3] + 1].T @ F[:, S[:3] + 1], rtol=0, atol=1e-12)


def test_upper_power_is_ten_power_iterations():
    """UPPER_KER restatement (ParaLanczos.cu:1484-1626) with the all-ones start:
    10 iterations of w = A v, b = ||w||, v = w / b; a lower estimate of ||A||_2
    that approaches it from below."""
    rng = np.random.default_rng(1)
    P = rng.standard_normal((80, 40))
    A = P.T @ P / 80
    v = np.ones(40) / np.sqrt(40)
    for _ in range(10):
        w = A @ v
        b = np.linalg.norm(w)
        v = w / b
    assert abs(O.upper_power(A) - b) <= 1e-12 * b
    assert O.upper_power(A) <= np.linalg.eigvalsh(A)[-1] * (1 + 1e-12)
