"""Multi-process host logic on CPU (gloo, world size 2): set-range sharding,
the RIP-sweep reduction, checkpoint/resume, and failure of a rank.

The per-set solver in these tests is the CPU oracle (the reference's per-set
algorithm restated), standing in for the GPU solve: what is under test is the
host-side sharding and reduction, which is identical for both solvers.
"""
import datetime
import math
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from paralanczos_b200.sweep import rip_sweep, shard_range

N, K, SEED = 96, 8, 5


def _matrix():
    rng = np.random.default_rng(3)
    Phi = rng.standard_normal((32, N)) / np.sqrt(32)
    return (Phi.T @ Phi).astype(np.float32)


def _oracle_solver():
    from oracle import oracle as O
    A = _matrix()

    def solve_chunk(first, count):
        _, idx = O.gen_stream(SEED, first, count, N, 0, K, K)
        r = O.batch(A, idx, k=K, nthreads=1)
        return r["delta"], r["err"]

    return solve_chunk


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, nsets, chunk, ckdir, mode, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=8))
    try:
        solver = _oracle_solver()
        if mode == "fail" and rank == 1:
            raise RuntimeError("planted failure of rank 1 before the reduction")
        ck = os.path.join(ckdir, "sweep-{rank}.json") if ckdir else None
        if mode == "partial":
            r = rip_sweep(solver, nsets, chunk=chunk, checkpoint=ck, max_chunks=1)
        else:
            r = rip_sweep(solver, nsets, chunk=chunk, checkpoint=ck)
        q.put((rank, "ok", r.delta, r.set_id, r.n_solved, r.n_failed))
    except Exception as e:  # noqa: BLE001 - reported to the parent
        q.put((rank, "error", type(e).__name__ + ": " + str(e)[:200], -1, 0, 0))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(world, nsets, chunk=16, ckdir=None, mode="normal"):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, nsets, chunk, ckdir, mode, q))
          for r in range(world)]
    for p in ps:
        p.start()
    out = {}
    for _ in range(world):
        item = q.get(timeout=120)
        out[item[0]] = item[1:]
    for p in ps:
        p.join(timeout=60)
    return out


def _single(nsets, chunk=16):
    return rip_sweep(_oracle_solver(), nsets, chunk=chunk)


def test_shard_range_partitions_exactly():
    for nsets in (0, 1, 7, 100, 101):
        for world in (1, 2, 3, 8):
            spans = [shard_range(nsets, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == nsets
            for a, b in zip(spans, spans[1:]):
                assert a[1] == b[0]
            sizes = [h - l for l, h in spans]
            assert max(sizes) - min(sizes) <= 1


def test_two_ranks_equal_single_process():
    ref = _single(64)
    out = _run(2, 64)
    assert all(v[0] == "ok" for v in out.values()), out
    for rank, (_, d, sid, solved, failed) in out.items():
        assert d == ref.delta and sid == ref.set_id
        assert solved == 64 and failed == 0


def test_checkpoint_resume_matches_uninterrupted():
    ref = _single(64)
    with tempfile.TemporaryDirectory() as d:
        part = _run(2, 64, chunk=8, ckdir=d, mode="partial")   # one chunk per rank, then stop
        assert all(v[0] == "ok" for v in part.values())
        assert sorted(os.listdir(d)) == ["sweep-0.json", "sweep-1.json"]
        full = _run(2, 64, chunk=8, ckdir=d)                   # resumes after the saved chunk
        for rank, (_, dl, sid, solved, _) in full.items():
            assert dl == ref.delta and sid == ref.set_id and solved == 64


def test_failed_rank_is_detected_by_the_others():
    out = _run(2, 64, mode="fail")
    assert out[1][0] == "error" and "planted failure" in out[1][1]
    # rank 0 waits in the all-gather and gets an error (timeout / peer closed)
    assert out[0][0] == "error"


def test_nan_sets_do_not_win():
    def solver(first, count):
        d = np.full(count, np.nan)
        e = np.full(count, 2, dtype=np.int32)   # PL_SET_NONFINITE
        if first == 0:
            d[3], e[3] = 0.25, 0
        return d, e
    r = rip_sweep(solver, 40, chunk=10)
    assert r.delta == 0.25 and r.set_id == 3 and r.n_solved == 1 and r.n_failed == 39
    r = rip_sweep(lambda f, c: (np.full(c, np.nan), np.full(c, 2, np.int32)), 10, chunk=5)
    assert math.isnan(r.delta) and r.set_id == -1
