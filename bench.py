#!/usr/bin/env python3
"""Benchmark: subset eigen-solves/s at k=64 (batched vs plain), one JSON line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2|c3|c4|c5]

The default workload (c2) is the headline configuration described below;
c1 (small, through the reference's C entry point), c3 (uneven k in one
launch), c4 (on-the-fly Gram) and c5 (serving) print their own JSON line with
the same keys (see bench_extra.py).

Workload (the configuration the headline metric is quoted on): Phi 1024x4096
with i.i.d. N(0, 1/1024) entries (numpy default_rng(0), stored FP32),
A = Phi^T Phi formed in FP64 and stored FP32 (64 MB; workloads.py, the same
bits in both arms); 1,000,000 index sets of k = 64 distinct
columns from the project's counter-based generator (seed 1); per set the
k-step Lanczos (FP32, FP64 alpha/beta, full reorthogonalisation) and FP64
Sturm bisection of lambda_min / lambda_max / delta_k.  Synthetic data: the
reference publishes no dataset.

A step = one pass of the batched form over all sets with inputs resident in
HBM.  The 256 MB index array exceeds L2; in addition a 256 MB buffer is written
between timed steps (outside the timed events) so A starts each step cold.

`e2e` is the same metric through the C ABI with HOST buffers (pl_solve_host:
H2D of A and the sets from pinned memory, solve, D2H of lambda_min,
lambda_max, delta_k, err) per step.  `plain` is the one-set-per-block form on
the same sets.  `accuracy` is the max and p99 relative error of lambda_min and
lambda_max against FP64 LAPACK dsyev over 2,000 sets spread over the
1,000,000 (every 500th).  `cpu_baseline` is the CPU oracle (the reference's per-set
algorithm restated in FP64, OpenMP over all host cores) on a bounded sample.

With N > 1 (torchrun, one rank per GPU) every rank solves its own 1,000,000
sets (set ids rank*1e6 ..): weak scaling, no data-path collective; the time is
the max over ranks.  --impl reference times the CPU oracle on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import workloads  # noqa: E402

METRIC = "subset eig-solves/s @k=64, err<=1e-5 vs FP64: plain vs batched; serve p50/p99"
N_COLS, M_ROWS, K, NSETS = workloads.C2["n"], workloads.C2["m"], workloads.C2["k"], workloads.C2["nsets"]
SEED_PHI, SEED_SETS = workloads.SEED_PHI, workloads.SEED_SETS
WORKLOAD = ("Phi 1024x4096 N(0,1/1024) seed 0 (numpy, FP32), A=Phi^T Phi FP32 64 MB; 1,000,000 sets "
            "k=64 (counter-based generator, seed 1); batched persistent form")
ACC_STRIDE = 500  # accuracy sample: every 500th set -> 2,000 of the 1,000,000


def flops_per_set(k: int) -> float:
    return 4.0 * k ** 3            # k matvecs (2k^3) + one full reorthogonalisation pass (2k^3)


def gather_bytes_per_set(k: int) -> float:
    return 4.0 * k * (k + 1) / 2 + 4.0 * k + 28.0


def dsyev_eigs(M) -> np.ndarray:
    """FP64 LAPACK dsyev eigenvalues (ascending) of a symmetric matrix."""
    from scipy.linalg import lapack
    w, _, info = lapack.dsyev(np.asarray(M, dtype=np.float64), compute_v=0)
    assert info == 0, info
    return w


def accuracy_vs_dsyev(A32, idx_np, k, lmin, lmax, sets):
    """Relative error of lambda_min / lambda_max against FP64 LAPACK dsyev of
    the same FP32 submatrix promoted to FP64, over the given set ids:
    {sets_checked, max, p99} (each set contributes its worse extreme)."""
    errs = np.empty(len(sets))
    for j, s in enumerate(sets):
        S = idx_np[s * k:(s + 1) * k]
        w = dsyev_eigs(A32[np.ix_(S, S)])
        errs[j] = max(abs(lmin[s] - w[0]) / abs(w[0]), abs(lmax[s] - w[-1]) / abs(w[-1]))
    return {"sets_checked": int(len(sets)), "max": float(errs.max()),
            "p99": float(np.percentile(errs, 99)), "bar": 1e-5}


# ----------------------------------------------------------------------------- clocks


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.rows.append([c.strip() for c in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ----------------------------------------------------------------------------- helpers


def profile_traffic(name: str):
    """dram bytes per launch from a committed ncu summary (profiles/<name>), or None."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            return json.load(open(p)), "measured"
        except Exception:
            pass
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_oracle_rate(A_np, idx_np, k, budget_s: float, nthreads: int = 0):
    """Sets/s of the CPU oracle on a bounded sample sized to ~budget_s seconds."""
    from oracle import oracle as O
    O.use_reference_tqlrat(True)
    cores = nthreads or os.cpu_count() or 1
    pilot = min(2000, len(idx_np) // k)
    t0 = time.perf_counter()
    O.batch(A_np, idx_np[:pilot * k], k=k, nthreads=cores)
    dt = time.perf_counter() - t0
    n = int(min(len(idx_np) // k, max(pilot, pilot * budget_s / max(dt, 1e-6))))
    t0 = time.perf_counter()
    O.batch(A_np, idx_np[:n * k], k=k, nthreads=cores)
    dt = time.perf_counter() - t0
    kind = "reference" if O.ref_lib() is not None else "port"
    return n / dt, n, cores, dt, kind


def lapack_rate(A64, idx, k, budget_s):
    """Sets/s of LAPACK dsyevr (extremes only, FP64) on the host, one set at a
    time, over a bounded sample; BLAS threads as the process has them."""
    from scipy.linalg import lapack
    n = len(idx) // k
    t0 = time.perf_counter()
    done = 0
    for s in range(n):
        S = idx[s * k:(s + 1) * k]
        w = lapack.dsyevr(A64[np.ix_(S, S)], compute_v=0, range="I", il=1, iu=1)[0]
        w = lapack.dsyevr(A64[np.ix_(S, S)], compute_v=0, range="I", il=k, iu=k)[0]
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    return done / (time.perf_counter() - t0), done


# ----------------------------------------------------------------------------- arms


def config_dict(ws: int) -> dict:
    return {"workload": WORKLOAD, "k": K, "sets_per_gpu": NSETS, "n": N_COLS,
            "l2": "256 MB index array per step exceeds L2; 256 MB L2 flush between steps",
            "parallelism": f"replicas x{ws}, set-range sharded" if ws > 1 else "single GPU"}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle as O
    A = np.array(workloads.c2_matrix()[1])  # the GPU arm's matrix, bit for bit
    cores = os.cpu_count() or 1
    sample = 4000
    _, idx = O.gen_stream(SEED_SETS, 0, sample, N_COLS, 0, K, K)
    O.use_reference_tqlrat(True)
    for _ in range(args.warmup):
        O.batch(A, idx[:200 * K], k=K, nthreads=cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.batch(A, idx, k=K, nthreads=cores)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * sum(times) / len(times)
    v = sample / (ms * 1e-3)
    kind = "reference" if O.ref_lib() is not None else "port"
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(ws),
        "sample": "the first 4,000 sets of the workload's set stream per step (the sets of rank 0)",
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": kind,
                         "sample": "the first 4,000 sets of the workload per step, OpenMP over all host cores; "
                                   "FP64 KER2 recurrence restated + TQLRAT/DET_TRIDIAG"
                                   + (" compiled from the reference source" if kind == "reference"
                                      else " restated")},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    from paralanczos_b200 import api
    from paralanczos_b200._lib import lib

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
        pg = dist

    def barrier():
        torch.cuda.synchronize()
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    A_np = np.array(workloads.c2_matrix()[1])
    A = torch.from_numpy(A_np).to(dev)
    first = rank * NSETS
    idx = api.gen_sets(SEED_SETS, first, NSETS, N_COLS, K)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    out = api.solve(A, idx, k=K)
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize()

    # accuracy on 2,000 sets spread over the run (FP64 dsyev on the CPU)
    acc = accuracy_vs_dsyev(A_np, idx.cpu().numpy(), K, out["lmin"].cpu().numpy(), out["lmax"].cpu().numpy(),
                            range(0, NSETS, ACC_STRIDE))
    acc["sample"] = f"every {ACC_STRIDE}th set of the {NSETS:,} (rank 0's sets)"

    for _ in range(args.warmup):
        api.solve(A, idx, k=K, out=out)
    barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    sampler = ClockSampler(local)
    with sampler:
        t0 = time.perf_counter()
        for i in range(args.steps):
            flush.fill_(float(i))                        # evict L2 (outside the timed events)
            evs[i][0].record(stream)
            api.solve(A, idx, k=K, out=out)
            evs[i][1].record(stream)
        barrier()
        wall = time.perf_counter() - t0
    step_ms = [a.elapsed_time(b) for a, b in evs]
    my_ms = sum(step_ms) / len(step_ms)
    t = torch.tensor([my_ms], device=dev, dtype=torch.float64)
    if pg is not None:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    ms = float(t.item())
    value = ws * NSETS / (ms * 1e-3)

    # plain one-set-per-block form on the same sets
    api.solve(A, idx, k=K, form="plain", out=out)
    barrier()
    pe = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(2)]
    for a, b in pe:
        flush.fill_(1.0)
        a.record(stream)
        api.solve(A, idx, k=K, form="plain", out=out)
        b.record(stream)
    barrier()
    plain_ms = sum(a.elapsed_time(b) for a, b in pe) / len(pe)
    api.solve(A, idx, k=K, out=out)

    # end to end through the C ABI with pinned host buffers
    A_h = A.cpu().pin_memory()
    idx_h = idx.cpu().pin_memory()
    outs_h = {n: torch.empty(NSETS, dtype=torch.float64 if n != "err" else torch.int32).pin_memory()
              for n in ("lmin", "lmax", "delta", "err")}
    L = lib()

    def e2e_call():
        rc = L.pl_solve_host(A_h.data_ptr(), N_COLS, N_COLS, idx_h.data_ptr(), None, NSETS, K, 0,
                             outs_h["lmin"].data_ptr(), outs_h["lmax"].data_ptr(),
                             outs_h["delta"].data_ptr(), outs_h["err"].data_ptr(), None, None)
        assert rc == 0, rc

    e2e_call()
    e2e_times = []
    for _ in range(max(2, min(args.steps, 5))):
        t1 = time.perf_counter()
        e2e_call()
        e2e_times.append(time.perf_counter() - t1)
    e2e_s = sum(e2e_times) / len(e2e_times)
    assert np.array_equal(outs_h["lmin"].numpy(), out["lmin"].cpu().numpy())
    h2d = A_h.numel() * 4 + idx_h.numel() * 4
    d2h = NSETS * (8 * 3 + 4)

    # the gather alone (pl_gather_blocks) on 200,000 of the sets
    gsets = 200_000
    gidx = idx[:gsets * K]
    gout = api.gather_blocks(A, gidx, K)
    ge = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(3)]
    for a, b in ge:
        flush.fill_(2.0)
        a.record(stream)
        api.gather_blocks(A, gidx, K, out=gout)
        b.record(stream)
    torch.cuda.synchronize()
    g_s = sum(a.elapsed_time(b) for a, b in ge) / len(ge) * 1e-3
    del gout
    g_read = gsets * (4.0 * K * (K + 1) / 2 + 4.0 * K) / g_s / 1e9
    g_write = gsets * 4.0 * K * K / g_s / 1e9
    g_elems = gsets * K * (K + 1) / 2 / g_s / 1e9          # random elements, G/s
    g_ceiling = api.gather_peak()                          # measured random-load ceiling, G/s

    peak_fp32 = api.fp32_peak()
    peaks, peak_src = measured_peaks()
    achieved = flops_per_set(K) * NSETS / (my_ms * 1e-3) / 1e12
    traffic = profile_traffic("k_sa_solve_k64_c2.md")
    gather_gbs = gather_bytes_per_set(K) * NSETS / (my_ms * 1e-3) / 1e9

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        idx_cpu = idx[:200_000 * K].cpu().numpy()
        rate, n, cores, dt, kind = cpu_oracle_rate(A_np, idx_cpu, K, args.cpu_budget)
        lr, ln = lapack_rate(A_np.astype(np.float64), idx_cpu, K, 5.0)
        cpu = {"value": rate, "unit": "solves/s", "cores": cores, "kind": kind,
               "sample": f"{n} sets of the workload ({dt:.1f} s), OpenMP over {cores} host threads; "
                         "FP64 KER2 recurrence restated + TQLRAT/DET_TRIDIAG"
                         + (" compiled from the reference source" if kind == "reference" else ""),
               "lapack_dsyevr": {"value": lr, "sets": ln, "note": "extremes only, one set per call, FP64"}}

    if rank == 0:
        bin_k = next(b for b in range(api.num_bins()) if api.bin_kmax(b) >= K)  # the bin k = 64 runs in
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "precision": "FP32 vectors and matvecs; FP64 alpha/beta accumulation and Sturm bisection",
            "config": config_dict(ws),
            "e2e": {"value": NSETS / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h),
                    "path": "pl_solve_host (C ABI, pinned host buffers: A copied in before the launch; the sets "
                            "read by the kernel from pinned host memory while it computes; results copied out)"},
            "gpu_launches": args.steps,
            "plain": {"value": NSETS / (plain_ms * 1e-3), "unit": "solves/s", "ms_per_step": plain_ms,
                      "form": "one set per thread block (PL_FORM_PLAIN)"},
            "batched_vs_plain": plain_ms / my_ms,
            "accuracy": acc,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak_fp32, "unit": "TFLOP/s",
                         "frac": achieved / peak_fp32, "traffic": traffic,
                         "kernel": api.tune_describe(bin_k, api.tune_get(bin_k))[1],
                         "peak_source": "FP32 FMA peak measured live by k_fma_peak (no FP32 figure in "
                                        "MEASURED_PEAKS.json)",
                         "algorithmic": "4k^3 FLOP per set (k matvecs + one reorthogonalisation pass)"},
            "roofline_gather": {"bound": "hbm", "achieved": gather_gbs, "peak": peaks.get("hbm_gbs"),
                                "unit": "GB/s", "frac": gather_gbs / peaks.get("hbm_gbs"),
                                "peak_source": peak_src,
                                "algorithmic": "4k(k+1)/2 + 4k + 28 bytes per set over the whole kernel"},
            "gather_only": {"sets": gsets, "ms": g_s * 1e3, "read_gbs": g_read, "write_gbs": g_write,
                            "frac_hbm": (g_read + g_write) / peaks.get("hbm_gbs"),
                            "random_gelems": g_elems, "ceiling_gelems": g_ceiling,
                            "frac_ceiling": g_elems / g_ceiling,
                            "ceiling": "uniformly random 4-byte loads from an L2-resident array, measured "
                                       "live (pl_gather_peak): each element is its own L1 request and sector",
                            "kernel": "k_gather_blocks (pl_gather_blocks): A[S,S] written as k x k blocks",
                            "algorithmic": "read 4k(k+1)/2 + 4k bytes, write 4k^2 bytes per set"},
            "clocks": sampler.summary(),
            "wall_s_timed": wall,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of CPU-baseline work")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5"])
    ap.add_argument("--rates", default="", help="c5: comma-separated request rates (1/s) to sweep")
    ap.add_argument("--requests", type=int, default=0, help="c5: requests per rate")
    args = ap.parse_args()
    if args.workload != "c2":
        import bench_extra
        return bench_extra.run(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
