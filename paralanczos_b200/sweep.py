"""RIP sweep: the largest delta_k over a family of index sets, sharded over ranks.

The reference stops at per-set eigenvalues and leaves the restricted-isometry
aggregate to its callers (README.md:2; the unused ``subseq`` bound fields in
ParaLanczos0.h:82-90).  Here a sweep over sets ``first .. first + nsets - 1`` of
a generator stream is split into contiguous per-rank ranges (set ``s`` depends
only on ``(seed, s)``, so no index data moves), each rank reduces its own
maximum and arg-max locally, and the only collective is one all-gather of
``(delta, set)`` per rank at the end.  Progress can be checkpointed per rank
and a sweep resumed by set range.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass


@dataclass
class SweepResult:
    delta: float       # max delta_k found (NaN if no set was solved)
    set_id: int        # the set that attains it (-1 if none)
    n_solved: int      # sets solved by all ranks
    n_failed: int      # sets with an error bit other than breakdown


def shard_range(nsets: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous, balanced [lo, hi) of the set range owned by `rank`."""
    base, extra = divmod(nsets, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _better(a: tuple[float, int], b: tuple[float, int]) -> bool:
    """Larger delta wins; ties go to the smaller set id (deterministic)."""
    if math.isnan(b[0]):
        return not math.isnan(a[0])
    if math.isnan(a[0]):
        return False
    return a[0] > b[0] or (a[0] == b[0] and a[1] < b[1])


def _load_ckpt(path: str | None):
    if path and os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return None


def _save_ckpt(path: str | None, state: dict) -> None:
    if not path:
        return
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(state, f)
    os.replace(tmp, path)


def rip_sweep(solve_chunk, nsets: int, first: int = 0, chunk: int = 1 << 20, group=None,
              checkpoint: str | None = None, max_chunks: int | None = None) -> SweepResult:
    """Max delta_k over sets first .. first+nsets-1, sharded over `group`.

    solve_chunk(first_set, count) -> (delta, err): per-set delta_k (float array)
    and status bits (int array) for `count` consecutive sets starting at global
    set id `first_set`.  On GPU this generates the sets on the device and calls
    pl_solve; any solver with that contract works.

    checkpoint: per-rank JSON file ("{rank}" is substituted); a rerun with the
    same arguments resumes after the last completed chunk.  max_chunks stops a
    rank early (the state is checkpointed), for resumable partial sweeps.
    """
    import numpy as np
    rank, world = 0, 1
    if group is not None or _dist_ready():
        import torch.distributed as dist
        rank, world = dist.get_rank(group), dist.get_world_size(group)
    lo, hi = shard_range(nsets, world, rank)
    ck = checkpoint.format(rank=rank) if checkpoint else None
    state = _load_ckpt(ck)
    key = {"first": first, "nsets": nsets, "world": world, "chunk": chunk}
    if state is None or state.get("key") != key:
        state = {"key": key, "next": lo, "delta": float("nan"), "set": -1, "solved": 0, "failed": 0}
    done_chunks = 0
    while state["next"] < hi:
        if max_chunks is not None and done_chunks >= max_chunks:
            break
        s0 = state["next"]
        cnt = min(chunk, hi - s0)
        delta, err = solve_chunk(first + s0, cnt)
        delta = np.asarray(delta, dtype=np.float64)
        err = np.asarray(err)
        ok = ((err & ~1) == 0) & np.isfinite(delta)
        state["solved"] += int(ok.sum())
        state["failed"] += int((~ok).sum())
        if ok.any():
            d = np.where(ok, delta, -np.inf)
            i = int(np.argmax(d))   # first maximum: smallest set id among ties
            cand = (float(d[i]), first + s0 + i)
            if _better(cand, (state["delta"], state["set"])):
                state["delta"], state["set"] = cand
        state["next"] = s0 + cnt
        done_chunks += 1
        _save_ckpt(ck, state)

    local = (state["delta"], state["set"], state["solved"], state["failed"])
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([local[0], float(local[1]), float(local[2]), float(local[3])],
                         dtype=torch.float64)
        if dist.get_backend(group) == "nccl":
            t = t.cuda()
        parts = [torch.zeros_like(t) for _ in range(world)]
        dist.all_gather(parts, t, group=group)
        best = (float("nan"), -1)
        solved = failed = 0
        for p in parts:
            p = p.cpu().tolist()
            if _better((p[0], int(p[1])), best):
                best = (p[0], int(p[1]))
            solved += int(p[2])
            failed += int(p[3])
        return SweepResult(best[0], best[1], solved, failed)
    return SweepResult(local[0], local[1], local[2], local[3])


def _dist_ready() -> bool:
    try:
        import torch.distributed as dist
        return dist.is_available() and dist.is_initialized()
    except Exception:
        return False


def gpu_solver(A, n: int, k: int, seed: int, stream=None):
    """solve_chunk for rip_sweep on the current GPU: sets generated on the
    device from (seed, set id), solved by the batched form."""
    from . import api

    def solve_chunk(first_set: int, count: int):
        idx = api.gen_sets(seed, first_set, count, n, k, device=A.device, stream=stream)
        out = api.solve(A, idx, k=k, stream=stream)
        return out["delta"].cpu().numpy(), out["err"].cpu().numpy()

    return solve_chunk
