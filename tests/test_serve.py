"""Serving (continuous batching) on the GPU.

A request's result must not depend on what it is batched with: requests are
solved alone and inside a mix of other matrices and k, and the results are
compared bit for bit, and against pl_solve on the same sets.  The batching
runs in device-resident request loops (a CUDA graph per loop under a
conditional WHILE node); a loop with nothing to do ends itself after a
bounded idle wait and is launched again by the next request.  Admission by
the HBM budget (which covers all of the server's device memory),
back-pressure of the pinned pool and per-set error reporting are checked
through the public API.
"""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mat(m, n, seed, kind="gauss"):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    Phi = torch.randn(m, n, generator=g, device="cuda", dtype=torch.float64) / m ** 0.5
    if kind == "corr":
        T = torch.eye(n, device="cuda", dtype=torch.float64)
        T += 0.3 * (torch.diag(torch.ones(n - 1, device="cuda", dtype=torch.float64), 1)
                    + torch.diag(torch.ones(n - 1, device="cuda", dtype=torch.float64), -1))
        Phi = Phi @ T
    return (Phi.T @ Phi).to(torch.float32).contiguous()


def _sets(rng, nsets, n, k):
    return np.stack([rng.choice(n, size=k, replace=False) for _ in range(nsets)]).astype(np.int32)


@pytest.fixture(scope="module")
def mats():
    return [_mat(256, 1024, 1), _mat(256, 1024, 2, "corr"), _mat(512, 2048, 3)]


def _solve_direct(A, S, k):
    import torch

    from paralanczos_b200 import api
    out = api.solve(A, torch.from_numpy(S.reshape(-1)).cuda(), k=k)
    return {key: v.cpu().numpy() for key, v in out.items()}


def _same(a, b):
    for key in ("lmin", "lmax", "delta", "err"):
        assert np.array_equal(a[key], b[key]), key


def test_alone_and_in_a_mix_are_bit_identical(mats):
    from paralanczos_b200.api import Server
    rng = np.random.default_rng(0)
    k0 = 48
    S0 = _sets(rng, 100, 1024, k0)
    with Server(budget_bytes=1 << 30, host_pool_bytes=256 << 20) as srv:
        ids = [srv.add_matrix(A) for A in mats]
        alone = srv.wait(srv.submit(ids[1], S0, k0), len(S0))
        # a burst of mixed requests with the same request in the middle
        reqs = []
        for i in range(40):
            if i == 20:
                reqs.append(("probe", srv.submit(ids[1], S0, k0), len(S0), None, None, None))
            m = int(rng.integers(0, 3))
            n = mats[m].shape[0]
            k = int(rng.choice([8, 16, 24, 33, 64, 100, 128, 160, 200, 256, 300]))
            ns = int(rng.integers(1, 120))
            S = _sets(rng, ns, n, k)
            reqs.append(("other", srv.submit(ids[m], S, k), ns, m, S, k))
        mixed = None
        others = []
        for tag, rid, ns, m, S, k in reqs:
            r = srv.wait(rid, ns)
            if tag == "probe":
                mixed = r
            else:
                others.append((r, m, S, k))
        st = srv.stats()
    _same(alone, mixed)
    _same(alone, _solve_direct(mats[1], S0, k0))
    # every other request equals the direct batched solve on its own
    for r, m, S, k in others:
        _same(r, _solve_direct(mats[m], S, k))
    assert st["completed"] == 42 and st["waves"] >= 1
    assert st["p99_s"] >= st["p50_s"] > 0


def test_results_match_dsyev(mats):
    from oracle import oracle as O
    from paralanczos_b200.api import Server
    rng = np.random.default_rng(1)
    A = mats[0].cpu().numpy().astype(np.float64)
    with Server(budget_bytes=1 << 30, host_pool_bytes=64 << 20) as srv:
        mid = srv.add_matrix(mats[0])
        for k in (8, 64, 128, 192):
            S = _sets(rng, 20, 1024, k)
            r = srv.wait(srv.submit(mid, S, k), len(S))
            assert ((r["err"] & ~1) == 0).all()
            for s in range(len(S)):
                w = O.dsyev_eigs(A[np.ix_(S[s], S[s])])
                assert abs(r["lmin"][s] - w[0]) <= 1e-5 * abs(w[0])
                assert abs(r["lmax"][s] - w[-1]) <= 1e-5 * abs(w[-1])


def test_admission_respects_the_budget(mats):
    from paralanczos_b200._lib import PLError
    from paralanczos_b200.api import Server
    rng = np.random.default_rng(2)
    budget = 384 << 20
    with Server(budget_bytes=budget, host_pool_bytes=1 << 30, max_waves=1) as srv:
        st0 = srv.stats()
        # every device byte of the server (arena, wave staging, scratch) is
        # inside the budget; what is left for indices is the arena
        assert st0["device_bytes"] <= budget
        arena = int(st0["arena_bytes"])
        mid = srv.add_matrix(mats[0])
        # each request's indices take a little over a third of the arena: at
        # most two fit at once, so admission waits for completions
        nsets = arena // 3 // (4 * 100) + 1
        batch = [_sets(rng, nsets, 1024, 100) for _ in range(5)]
        ids = [srv.submit(mid, S, 100) for S in batch]
        res = [srv.wait(i, nsets, 300.0) for i in ids]
        st = srv.stats()
        assert st["arena_peak"] <= arena
        assert st["arena_peak"] >= 2 * nsets * 400
        for S, r in zip(batch[:2], res[:2]):
            _same(r, _solve_direct(mats[0], S, 100))
        # a request that can never fit is refused up front
        with pytest.raises(PLError):
            srv.submit(mid, np.zeros(arena // 4 + 64, dtype=np.int32), 64)
    # a budget that does not even hold the server's staging is refused
    with pytest.raises(PLError):
        Server(budget_bytes=8 << 20, host_pool_bytes=1 << 20)


def test_idle_loop_ends_and_restarts(mats, monkeypatch):
    """With nothing to do a request loop waits at most PL_SERVE_IDLE_MS on the
    device and then ends (its graph finishes with status "idle"); the next
    request launches it again and is served."""
    import time

    from paralanczos_b200.api import Server
    monkeypatch.setenv("PL_SERVE_IDLE_MS", "5")
    rng = np.random.default_rng(9)
    with Server(budget_bytes=1 << 30, host_pool_bytes=64 << 20, max_waves=1) as srv:
        mid = srv.add_matrix(mats[0])
        S1 = _sets(rng, 50, 1024, 32)
        r1 = srv.wait(srv.submit(mid, S1, 32), 50)
        time.sleep(0.3)
        st = srv.stats()
        assert st["loop_launches"] >= 1
        assert st["idle_exits"] == st["loop_launches"]
        assert st["loops_running"] == 0
        S2 = _sets(rng, 50, 1024, 32)
        r2 = srv.wait(srv.submit(mid, S2, 32), 50)
        st2 = srv.stats()
        assert st2["loop_launches"] == st["loop_launches"] + 1
        _same(r1, _solve_direct(mats[0], S1, 32))
        _same(r2, _solve_direct(mats[0], S2, 32))


def test_large_request_split_over_waves_is_exact(mats, monkeypatch):
    """With short waves a large request runs as many pieces; the result is the
    same as one direct solve, and a small request submitted after it
    finishes first."""
    import time

    from paralanczos_b200.api import Server
    rng = np.random.default_rng(7)
    # ~3.2 us of estimated whole-GPU work per set of k = 200: 6.4 ms for the
    # request, so 0.2 ms waves cut it into some 30 pieces
    monkeypatch.setenv("PL_SERVE_WAVE_MS", "0.2")
    S = _sets(rng, 2000, 1024, 200)
    with Server(budget_bytes=1 << 30, host_pool_bytes=64 << 20) as srv:
        mid = srv.add_matrix(mats[0])
        r = srv.wait(srv.submit(mid, S, 200), len(S))
        assert srv.stats()["waves"] >= 20
        _same(r, _solve_direct(mats[0], S, 200))
    monkeypatch.delenv("PL_SERVE_WAVE_MS")
    big = _sets(rng, 1500, 2048, 500)
    small = _sets(rng, 5, 2048, 16)
    with Server(budget_bytes=1 << 30, host_pool_bytes=64 << 20) as srv:
        mid = srv.add_matrix(mats[2])
        rb = srv.submit(mid, big, 500)
        time.sleep(0.005)
        rs = srv.submit(mid, small, 16)
        out_s = srv.wait(rs, 5)
        out_b = srv.wait(rb, 1500)
        assert out_s["latency_s"] < out_b["latency_s"]
        _same(out_s, _solve_direct(mats[2], small, 16))


def test_pinned_pool_backpressure(mats):
    from paralanczos_b200.api import Server
    rng = np.random.default_rng(3)
    with Server(budget_bytes=1 << 30, host_pool_bytes=300_000) as srv:
        mid = srv.add_matrix(mats[0])
        S = _sets(rng, 400, 1024, 64)      # ~110 KB of pinned staging each
        first = [srv.try_submit(mid, S, 64) for _ in range(4)]
        assert first[0] is not None and first[1] is not None
        assert first[3] is None            # pool full: refused, not queued
        for rid in first:
            if rid is not None:
                srv.wait(rid, 400)
        again = srv.try_submit(mid, S, 64)
        assert again is not None
        srv.wait(again, 400)


def test_bad_index_and_bad_arguments(mats):
    from paralanczos_b200._lib import PLError
    from paralanczos_b200.api import Server
    rng = np.random.default_rng(4)
    with Server(budget_bytes=1 << 30, host_pool_bytes=16 << 20) as srv:
        mid = srv.add_matrix(mats[0])
        S = _sets(rng, 5, 1024, 16)
        S[3, 2] = 5000
        r = srv.wait(srv.submit(mid, S, 16), 5)
        assert r["err"][3] == 4 and np.isnan(r["lmin"][3])
        assert ((r["err"][[0, 1, 2, 4]] & ~1) == 0).all()
        with pytest.raises(PLError):
            srv.submit(mid, np.zeros(2000, dtype=np.int32), 2000)   # k > n
        with pytest.raises(PLError):
            srv.submit(7, S, 16)                                     # unknown matrix
        with pytest.raises(PLError):
            srv.wait(123456, 1, 0.01)                                # unknown request


def test_many_client_threads(mats):
    from paralanczos_b200.api import Server
    errors = []
    with Server(budget_bytes=1 << 30, host_pool_bytes=128 << 20) as srv:
        ids = [srv.add_matrix(A) for A in mats]

        def client(seed):
            rng = np.random.default_rng(100 + seed)
            try:
                for _ in range(6):
                    m = int(rng.integers(0, 3))
                    k = int(rng.choice([16, 64, 130]))
                    S = _sets(rng, int(rng.integers(1, 60)), mats[m].shape[0], k)
                    r = srv.wait(srv.submit(ids[m], S, k), len(S))
                    if not ((r["err"] & ~1) == 0).all():
                        errors.append(("err bits", seed))
            except Exception as e:  # noqa: BLE001 - collected for the assertion
                errors.append(repr(e))

        th = [threading.Thread(target=client, args=(i,)) for i in range(6)]
        for t in th:
            t.start()
        for t in th:
            t.join(timeout=120)
        assert srv.stats()["completed"] == 36
    assert not errors, errors
