"""Workloads c1 (small, drop-in path), c3 (uneven k), c4 (on-the-fly Gram) and
c5 (serving) of bench.py.

Each prints one JSON line with the keys of the headline line (metric, value,
unit, ms_per_step, e2e, roofline, cpu_baseline, clocks, gpu_launches, ...).

  c1  Phi 128x512 N(0,1/128) (seed 0), A = Phi^T Phi (512 x 512); 10,000 sets
      of k=16 (generator seed 1) through the reference's C entry point
      calculate_subeigs3 (host FP64 matrix in, all 16 eigenvalues and the
      determinant out), beside the batched and plain forms on device buffers;
      error vs dsyev, CPU oracle and LAPACK dsyevr timed beside it.
  c3  Phi 1024x4096 N(0,1/1024) (seed 0), A = Phi^T Phi FP32; 300,000 sets with
      k in {8,16,24,32,48,64,96,128,192,256}, P(k) ~ 1/k (the library's host
      generator, seed 1); one binned launch per step (device counting sort by k,
      per-bin persistent kernels, CUDA graph); per-k error vs dsyev.
  c4  Phi 2048x16384 stored FP32, N(0,1/2048) (value) and Rademacher
      +-1/sqrt(2048) (reported beside it); A never formed: A[S,S] = Phi_S^T Phi_S
      on the tensor cores per set; 500,000 sets of k=128; error vs dsyev on
      2,000 sampled sets (FP64 Gram of the FP32 frame).
  c5  four device-resident matrices (Gaussian 1024x4096, Rademacher 1024x4096,
      Gaussian 2048x16384, correlated 1024x4096 Phi = G (I + 0.3 T), T with
      ones on the first off-diagonals); open-loop Poisson request streams at
      swept rates; a request names a matrix (uniform), k uniform in [8, 512]
      and 1-4096 sets (log-uniform); the server (continuous batching, HBM
      budget) against one synchronous pl_solve call per request in arrival
      order (the plain per-call drop-in), p50/p99 latency and solves/s each.
Synthetic data throughout: the reference publishes no dataset.
"""
from __future__ import annotations

import json
import math
import os
import threading
import time

import numpy as np

import bench as B
import workloads as W

KV_C3 = (8, 16, 24, 32, 48, 64, 96, 128, 192, 256)


def _line(args, metric_value, ms, workload, extra):
    line = {"metric": B.METRIC, "value": metric_value, "unit": "solves/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "precision": "FP32 vectors and matvecs; FP64 alpha/beta accumulation and Sturm bisection",
            "data": "synthetic", "config": {"workload": workload}}
    line.update(extra)
    return line


def _timed_steps(fn, steps, warmup, flush, stream):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    sampler = B.ClockSampler(torch.cuda.current_device())
    with sampler:
        for i in range(steps):
            flush.fill_(float(i))
            evs[i][0].record(stream)
            fn()
            evs[i][1].record(stream)
        torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in evs]
    return sum(ms) / len(ms), sampler.summary()


# ----------------------------------------------------------------------------- c1


def run_c1(args):
    import torch

    from oracle import oracle as O
    from paralanczos_b200 import api
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n, k, nsets = W.C1["n"], W.C1["k"], W.C1["nsets"]
    A64, A32 = W.c1_matrix()
    A64 = np.array(A64)
    _, idx_h = api.gen_stream_host(B.SEED_SETS, 0, nsets, n, 0, k, k)
    idx_h = np.ascontiguousarray(idx_h, dtype=np.int32)
    eig = np.zeros(nsets * k)
    det = np.zeros(nsets)
    api.calculate_subeigs3(A64, nsets * k, n, eig, det, idx_h, k)
    t = []
    for _ in range(max(args.steps, 3)):
        t0 = time.perf_counter()
        rc = api.calculate_subeigs3(A64, nsets * k, n, eig, det, idx_h, k)
        t.append(time.perf_counter() - t0)
        assert rc == 0
    dropin_s = sum(t) / len(t)
    # device forms on the same sets
    A = torch.from_numpy(np.array(A32)).to(dev)
    idx = torch.from_numpy(idx_h).to(dev)
    flush = torch.empty(256 << 18, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    out = api.solve(A, idx, k=k)
    ms, clocks = _timed_steps(lambda: api.solve(A, idx, k=k, out=out), args.steps, args.warmup, flush, stream)
    outp = api.solve(A, idx, k=k, form="plain")
    ms_plain, _ = _timed_steps(lambda: api.solve(A, idx, k=k, form="plain", out=outp), 3, 2, flush, stream)
    lmin = out["lmin"].cpu().numpy()
    lmax = out["lmax"].cpu().numpy()
    errs = np.empty(2 * nsets)
    worst_all = 0.0
    for s in range(nsets):
        S = idx_h[s * k:(s + 1) * k]
        w = B.dsyev_eigs(A64[np.ix_(S, S)])
        errs[2 * s] = abs(lmin[s] - w[0]) / w[0]
        errs[2 * s + 1] = abs(lmax[s] - w[-1]) / w[-1]
        worst_all = max(worst_all, np.max(np.abs(eig[s * k:(s + 1) * k] - w)) / np.max(np.abs(w)))
    worst = float(np.max(errs))
    cpu = None
    if not args.no_cpu:
        O.use_reference_tqlrat(True)
        cores = os.cpu_count() or 1
        reps = 0
        t0 = time.perf_counter()
        while reps < 1 or time.perf_counter() - t0 < min(2.0, args.cpu_budget):
            O.batch(A64, idx_h, k=k, nthreads=cores)
            reps += 1
        dt = (time.perf_counter() - t0) / reps
        kind = "reference" if O.ref_lib() is not None else "port"
        lr, ln = B.lapack_rate(A64, idx_h, k, min(5.0, args.cpu_budget))
        cpu = {"value": nsets / dt, "unit": "solves/s", "cores": cores, "kind": kind,
               "sample": f"all {nsets} sets, {reps} passes ({dt * 1e3:.1f} ms each), FP64 KER2 recurrence "
                         f"restated + TQLRAT/DET_TRIDIAG, OpenMP over {cores} threads",
               "lapack_dsyevr": {"value": lr, "sets": ln, "note": "extremes only, one set per call"}}
    line = _line(args, nsets / (ms * 1e-3), ms,
                 "c1: Phi 128x512 N(0,1/128) seed 0, A 512x512; 10,000 sets k=16 (seed 1); batched form on "
                 "device buffers; the reference's C entry point timed beside it", {
                     "e2e": {"value": nsets / dropin_s, "unit": "solves/s",
                             "h2d_bytes_per_step": int(A64.nbytes + idx_h.nbytes),
                             "d2h_bytes_per_step": int(eig.nbytes + det.nbytes),
                             "path": "calculate_subeigs3 (reference C entry point: host FP64 matrix in, all "
                                     "eigenvalues and determinants out)"},
                     "gpu_launches": args.steps,
                     "plain": {"value": nsets / (ms_plain * 1e-3), "ms_per_step": ms_plain},
                     "accuracy": {"sets_checked": nsets, "max_rel_err_vs_dsyev_extremes": worst,
                                  "p99_rel_err_vs_dsyev_extremes": float(np.percentile(errs, 99)),
                                  "max_err_all_eigenvalues_drop_in": worst_all},
                     "roofline": {"bound": "fp32", "achieved": 4.0 * k ** 3 * nsets / (ms * 1e-3) / 1e12,
                                  "peak": api.fp32_peak(), "unit": "TFLOP/s", "traffic": None,
                                  "note": "10,000 sets fill the GPU for ~0.1 ms: launch-bound"},
                     "clocks": clocks})
    line["roofline"]["frac"] = line["roofline"]["achieved"] / line["roofline"]["peak"]
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- c3


def run_c3(args):
    import torch

    from oracle import oracle as O
    from paralanczos_b200 import api
    from paralanczos_b200._lib import lib
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    nsets, n = W.C3["nsets"], W.C3["n"]
    A = torch.from_numpy(np.array(W.c2_matrix()[1])).to(dev)
    off_h, idx_h = api.gen_stream_host(B.SEED_SETS, 0, nsets, n, kdist=1)
    ks = np.diff(off_h)
    idx = torch.from_numpy(idx_h).to(dev)
    off = torch.from_numpy(off_h).to(dev)
    flush = torch.empty(256 << 18, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    out = api.solve(A, idx, offsets=off)
    torch.cuda.synchronize()
    ms, clocks = _timed_steps(lambda: api.solve(A, idx, offsets=off, out=out), args.steps, args.warmup,
                              flush, stream)
    flops = float(np.sum(4.0 * ks.astype(np.float64) ** 3))
    achieved = flops / (ms * 1e-3) / 1e12
    peak = api.fp32_peak()
    # per-k error vs dsyev (16 sets per k value)
    A_np = A.cpu().numpy()
    A64 = A_np.astype(np.float64)
    lmin = out["lmin"].cpu().numpy()
    lmax = out["lmax"].cpu().numpy()
    err = out["err"].cpu().numpy()
    # per k: max and p99 of the relative error of lambda_min and lambda_max
    # against FP64 dsyev over 200 sets of that k spread over the stream
    per_k = {}
    for kv in KV_C3:
        ids = np.nonzero(ks == kv)[0]
        sel = ids[np.linspace(0, len(ids) - 1, min(200, len(ids))).astype(np.int64)]
        errs = []
        for s in sel:
            S = idx_h[off_h[s]:off_h[s + 1]]
            w = B.dsyev_eigs(A64[np.ix_(S, S)])
            errs += [abs(lmin[s] - w[0]) / abs(w[0]), abs(lmax[s] - w[-1]) / abs(w[-1])]
        per_k[str(kv)] = {"sets": int(len(ids)), "checked": int(len(sel)), "max_rel_err": float(np.max(errs)),
                          "p99_rel_err": float(np.percentile(errs, 99))}
    # end to end through the C ABI with pinned host buffers
    A_h = A.cpu().pin_memory()
    idx_p = torch.from_numpy(idx_h).pin_memory()
    off_p = torch.from_numpy(off_h).pin_memory()
    outs = {k: torch.empty(nsets, dtype=torch.float64 if k != "err" else torch.int32).pin_memory()
            for k in ("lmin", "lmax", "delta", "err")}
    L = lib()

    def e2e():
        rc = L.pl_solve_host(A_h.data_ptr(), n, n, idx_p.data_ptr(), off_p.data_ptr(), nsets, 0, 0,
                             outs["lmin"].data_ptr(), outs["lmax"].data_ptr(), outs["delta"].data_ptr(),
                             outs["err"].data_ptr(), None, None)
        assert rc == 0, rc
    e2e()
    t = []
    for _ in range(3):
        t0 = time.perf_counter()
        e2e()
        t.append(time.perf_counter() - t0)
    e2e_s = sum(t) / len(t)
    assert np.array_equal(outs["lmin"].numpy(), lmin)
    cpu = None
    if not args.no_cpu:
        O.use_reference_tqlrat(True)
        cores = os.cpu_count() or 1
        pilot = 2000
        t0 = time.perf_counter()
        O.batch(A_np, idx_h[:off_h[pilot]], offsets=off_h[:pilot + 1], nthreads=cores)
        dt = time.perf_counter() - t0
        m = int(min(nsets, max(pilot, pilot * args.cpu_budget / max(dt, 1e-6))))
        t0 = time.perf_counter()
        O.batch(A_np, idx_h[:off_h[m]], offsets=off_h[:m + 1], nthreads=cores)
        dt = time.perf_counter() - t0
        kind = "reference" if O.ref_lib() is not None else "port"
        cpu = {"value": m / dt, "unit": "solves/s", "cores": cores, "kind": kind,
               "sample": f"first {m} sets of the stream ({dt:.1f} s), OpenMP over {cores} threads"}
    line = _line(args, nsets / (ms * 1e-3), ms,
                 "c3: Phi 1024x4096 N(0,1/1024) seed 0, A FP32; 300,000 sets, k in {8..256} P~1/k "
                 "(seed 1); binned by k on the device, one CUDA graph per step", {
                     "e2e": {"value": nsets / e2e_s, "unit": "solves/s",
                             "h2d_bytes_per_step": int(A_h.numel() * 4 + idx_p.numel() * 4 + off_p.numel() * 8),
                             "d2h_bytes_per_step": int(nsets * 28), "path": "pl_solve_host, CSR offsets"},
                     "gpu_launches": args.steps * (4 + api.num_bins()),
                     "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                                  "frac": achieved / peak, "traffic": None,
                                  "algorithmic": "sum over sets of 4k^3 FLOP"},
                     "per_k": per_k, "mean_k": float(ks.mean()),
                     "err_bits_nonbreakdown": int(np.sum((err & ~1) != 0)),
                     "clocks": clocks})
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- c4


def _c4_frame(kind, dev):
    import torch
    return torch.from_numpy(W.c4_frame("gauss" if kind == "gauss" else "rademacher")).to(dev)


def _c4_accuracy(Phi, idx, out, k, nsample=2000):
    import torch

    nsets = idx.numel() // k
    step = max(1, nsets // nsample)
    sel = torch.arange(0, nsets, step, device=Phi.device)[:nsample]
    S = idx.view(nsets, k)[sel]
    lmin = out["lmin"][sel].cpu().numpy()
    lmax = out["lmax"][sel].cpu().numpy()
    P64 = Phi.double()
    worst = 0.0
    errs = []
    for c0 in range(0, len(sel), 200):
        Sc = S[c0:c0 + 200].long()
        X = P64[:, Sc].permute(1, 0, 2)                      # (b, m, k)
        G = torch.bmm(X.transpose(1, 2), X).cpu().numpy()   # FP64 Gram of the FP32 frame
        for j in range(G.shape[0]):
            w = B.dsyev_eigs(G[j])
            e = max(abs(lmin[c0 + j] - w[0]) / abs(w[0]), abs(lmax[c0 + j] - w[-1]) / abs(w[-1]))
            errs.append(e)
            worst = max(worst, e)
    return worst, float(np.percentile(errs, 99)), len(errs)


def run_c4(args):
    import torch

    from oracle import oracle as O
    from paralanczos_b200 import api
    from paralanczos_b200.api import GramFrame
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    m, n, k, nsets = 2048, 16384, 128, 500_000
    flush = torch.empty(256 << 18, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    idx = api.gen_sets(B.SEED_SETS, 0, nsets, n, k)
    res = {}
    for kind in ("gauss", "rad"):
        Phi = _c4_frame(kind, dev)
        t0 = time.perf_counter()
        gf = GramFrame(Phi)
        torch.cuda.synchronize()
        prep_s = time.perf_counter() - t0
        out = gf.solve(idx, k)
        torch.cuda.synchronize()
        ms, clocks = _timed_steps(lambda: gf.solve(idx, k, out=out), args.steps if kind == "gauss" else 2,
                                  args.warmup if kind == "gauss" else 1, flush, stream)
        worst, p99, nchk = _c4_accuracy(Phi, idx, out, k)
        # the Gram kernel alone on 32,768 sets (blocks written to HBM)
        sub = idx[:32768 * k]
        gf.blocks(sub, k)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        gms = []
        for _ in range(3):
            flush.fill_(0.0)
            e0.record(stream)
            gf.blocks(sub, k)
            e1.record(stream)
            torch.cuda.synchronize()
            gms.append(e0.elapsed_time(e1))
        gram_ms = sum(gms) / len(gms)
        res[kind] = dict(ms=ms, clocks=clocks, worst=worst, p99=p99, nchk=nchk, prep_s=prep_s,
                         gram_ms=gram_ms, err_bits=int(((out["err"] & ~1) != 0).sum().item()))
        if kind == "gauss":
            Phi_keep = Phi.cpu()
        del gf, out, Phi
        torch.cuda.empty_cache()
    r = res["gauss"]
    peaks, src = B.measured_peaks()
    useful = 2.0 * m * k * k * 32768
    tensor_tf = 3 * useful / (r["gram_ms"] * 1e-3) / 1e12
    gather_gbs = 32768 * m * k * 4 / (r["gram_ms"] * 1e-3) / 1e9
    lz_flops = 4.0 * k ** 3 * nsets
    lz_ms = r["ms"] - r["gram_ms"] * nsets / 32768
    peak32 = api.fp32_peak()
    # end to end: host frame and host sets in, host results out, per step
    Phi_h = Phi_keep.pin_memory()
    idx_h = idx.cpu().pin_memory()
    outs_h = {kk: torch.empty(nsets, dtype=torch.float64 if kk != "err" else torch.int32).pin_memory()
              for kk in ("lmin", "lmax", "delta", "err")}

    def e2e():
        Pd = Phi_h.to(dev, non_blocking=True)
        gfe = GramFrame(Pd)
        idd = idx_h.to(dev, non_blocking=True)
        o = gfe.solve(idd, k)
        for kk in outs_h:
            outs_h[kk].copy_(o[kk], non_blocking=True)
        torch.cuda.synchronize()
    e2e()
    t = []
    for _ in range(2):
        t0 = time.perf_counter()
        e2e()
        t.append(time.perf_counter() - t0)
    e2e_s = sum(t) / len(t)
    cpu = None
    if not args.no_cpu:
        # FP64 Gram (BLAS over all threads) + the oracle's per-set Lanczos/TQLRAT
        O.use_reference_tqlrat(True)
        cores = os.cpu_count() or 1
        P = Phi_keep.numpy().astype(np.float64)
        S = idx[:2000 * k].view(2000, k).cpu().numpy()
        t0 = time.perf_counter()
        for s in range(2000):
            X = P[:, S[s]]
            G = X.T @ X
            O.batch(G, np.arange(k, dtype=np.int32), k=k, nthreads=1)
            if time.perf_counter() - t0 > args.cpu_budget:
                break
        dt = time.perf_counter() - t0
        done = s + 1
        kind = "reference" if O.ref_lib() is not None else "port"
        cpu = {"value": done / dt, "unit": "solves/s", "cores": cores, "kind": kind,
               "sample": f"{done} sets ({dt:.1f} s): FP64 Gram by BLAS + per-set oracle Lanczos/TQLRAT; "
                         "rate extrapolated to the 500,000-set workload"}
    line = _line(args, nsets / (r["ms"] * 1e-3), r["ms"],
                 "c4: Phi 2048x16384 FP32 N(0,1/2048) seed 0 (Rademacher beside it), A never formed; "
                 "500,000 sets k=128 (seed 1); A[S,S] on tcgen05 (bf16 split, FP32 accumulate) then "
                 "Lanczos FP32 / FP64 scalars", {
                     "e2e": {"value": nsets / e2e_s, "unit": "solves/s",
                             "h2d_bytes_per_step": int(Phi_h.numel() * 4 + idx_h.numel() * 4),
                             "d2h_bytes_per_step": int(nsets * 28),
                             "path": "host frame + host sets -> GramFrame -> solve -> host results"},
                     "gpu_launches": args.steps * (2 * 16 + 1),
                     "roofline": {"bound": "fp32", "achieved": lz_flops / (lz_ms * 1e-3) / 1e12, "peak": peak32,
                                  "unit": "TFLOP/s", "frac": lz_flops / (lz_ms * 1e-3) / 1e12 / peak32,
                                  "traffic": None, "kernel": "Lanczos k=128 on the formed blocks "
                                  "(the dominant kernel: step time minus the Gram kernel's)"},
                     "roofline_gram": {"bound": "tensor", "achieved": tensor_tf,
                                       "traffic_8192_sets": B.profile_traffic("k_gram_c4.md"),
                                       "peak": peaks.get("bf16_tflops"), "unit": "TFLOP/s",
                                       "frac": tensor_tf / peaks.get("bf16_tflops"), "peak_source": src,
                                       "useful_tflops": useful / (r["gram_ms"] * 1e-3) / 1e12,
                                       "gather_gbs": gather_gbs,
                                       "gather_frac_hbm": gather_gbs / peaks.get("hbm_gbs"),
                                       "algorithmic": "3 x 2 M k^2 FLOP per set on the tensor pipe "
                                                      "(useful 2 M k^2); 4 M k bytes of bf16 pieces per set",
                                       "ms_32768_sets": r["gram_ms"]},
                     "accuracy": {"gauss": {"sets_checked": r["nchk"], "max_rel_err_vs_dsyev": r["worst"],
                                            "p99_rel_err": r["p99"]},
                                  "rademacher": {"sets_checked": res["rad"]["nchk"],
                                                 "max_rel_err_vs_dsyev": res["rad"]["worst"],
                                                 "p99_rel_err": res["rad"]["p99"]}},
                     "rademacher": {"value": nsets / (res["rad"]["ms"] * 1e-3), "ms_per_step": res["rad"]["ms"]},
                     "prepare_s": r["prep_s"], "err_bits_nonbreakdown": r["err_bits"],
                     "clocks": r["clocks"]})
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- c5


def _c5_matrices(dev):
    import torch
    out = []
    for label, m, n, kind, seed in W.C5_MATRICES:
        # the frame from workloads.frame (host, seeded); its FP64 Gram on the GPU
        Phi = torch.from_numpy(W.frame(m, n, seed, kind)).to(dev).double()
        A = (Phi.T @ Phi).to(torch.float32).contiguous()
        del Phi
        out.append((label, A))
        torch.cuda.synchronize()
    return out


def _c5_stream(rate, nreq, mats, seed):
    from paralanczos_b200 import api
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    for i in range(nreq):
        t += rng.exponential(1.0 / rate)
        mid = int(rng.integers(0, len(mats)))
        n = mats[mid][1].shape[0]
        k = int(rng.integers(8, 513))
        k = min(k, n)
        ns = int(math.floor(math.exp(rng.uniform(0.0, math.log(4097.0)))))
        ns = max(1, min(4096, ns))
        _, idx = api.gen_stream_host(seed * 1000003 + i, 0, ns, n, 0, k, k)
        reqs.append(dict(t=t, mat=mid, k=k, nsets=ns, idx=idx))
    return reqs


def _serve_ours(srv, ids, reqs):
    """Open loop: submit at each arrival time.  Latency = the server's own
    submit-to-completion time plus any delay of the submit past the arrival."""
    rids = [None] * len(reqs)
    late = [0.0] * len(reqs)
    t0 = time.perf_counter() + 0.05
    ready = threading.Semaphore(0)

    def submitter():
        for i, r in enumerate(reqs):
            dt = t0 + r["t"] - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            late[i] = max(0.0, time.perf_counter() - (t0 + r["t"]))
            while True:
                rid = srv.try_submit(ids[r["mat"]], r["idx"], r["k"])
                if rid is not None:
                    break
                time.sleep(0.0005)
            rids[i] = rid
            ready.release()

    th = threading.Thread(target=submitter)
    th.start()
    lat = []
    for i, r in enumerate(reqs):
        ready.acquire()
        out = srv.wait(rids[i], r["nsets"], timeout_s=600.0)
        lat.append(out["latency_s"] + late[i])
    th.join()
    return lat


def _serve_plain(mats, reqs):
    """One synchronous pl_solve call per request in arrival order."""
    import torch

    from paralanczos_b200 import api
    dev = mats[0][1].device
    lat = []
    t0 = time.perf_counter() + 0.05
    for r in reqs:
        dt = t0 + r["t"] - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        idx = torch.from_numpy(r["idx"]).to(dev)
        form = "plain" if r["k"] <= 128 else "batched"
        o = api.solve(mats[r["mat"]][1], idx, k=r["k"], form=form)
        _ = [o[kk].cpu() for kk in ("lmin", "lmax", "delta", "err")]
        lat.append(time.perf_counter() - (t0 + r["t"]))
    return lat


def _pct(x, p):
    return float(np.percentile(np.asarray(x), p))


def run_c5(args):
    import torch

    from paralanczos_b200.api import Server
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    mats = _c5_matrices(dev)
    nreq = args.requests or 80
    with Server(budget_bytes=2 << 30, host_pool_bytes=1 << 30, max_waves=4) as srv:
        ids = [srv.add_matrix(A) for _, A in mats]
        # warm-up: every bin's kernel loaded once
        warm = [dict(t=0.0, mat=0, k=kk, nsets=64, idx=None) for kk in (8, 16, 32, 64, 128, 192, 256, 384, 512)]
        from paralanczos_b200 import api
        for w in warm:
            _, w["idx"] = api.gen_stream_host(7, 0, 64, 4096, 0, w["k"], w["k"])
            srv.wait(srv.submit(ids[0], w["idx"], w["k"]), 64)
        # capacity: the whole stream submitted at once (closed burst)
        cal = _c5_stream(1e6, 40, mats, 5)
        srv.reset_stats()
        t0 = time.perf_counter()
        rids = [srv.submit(ids[r["mat"]], r["idx"], r["k"]) for r in cal]
        for r, rid in zip(cal, rids):
            srv.wait(rid, r["nsets"], timeout_s=600)
        cap_s = time.perf_counter() - t0
        cap = len(cal) / cap_s
        cal_sets = sum(r["nsets"] for r in cal)
        # the same burst through one synchronous call per request
        _serve_plain(mats, [dict(r, t=0.0) for r in cal[:4]])   # warm-up
        t0 = time.perf_counter()
        _serve_plain(mats, [dict(r, t=0.0) for r in cal])
        cap_plain_s = time.perf_counter() - t0
        rates = [float(x) for x in args.rates.split(",") if x] or [0.25 * cap, 0.5 * cap, 0.8 * cap]
        sweep = []
        for ri, rate in enumerate(rates):
            reqs = _c5_stream(rate, nreq, mats, 11 + ri)
            sets = sum(r["nsets"] for r in reqs)
            srv.reset_stats()
            t0 = time.perf_counter()
            lat = _serve_ours(srv, ids, reqs)
            span = time.perf_counter() - t0
            st = srv.stats()
            t0 = time.perf_counter()
            lat_p = _serve_plain(mats, reqs)
            span_p = time.perf_counter() - t0
            sweep.append({
                "rate_req_s": rate, "requests": nreq, "sets": sets,
                "served": {"p50_ms": 1e3 * _pct(lat, 50), "p99_ms": 1e3 * _pct(lat, 99),
                           "server_p50_ms": 1e3 * st["p50_s"], "server_p99_ms": 1e3 * st["p99_s"],
                           "solves_s": sets / span, "waves": int(st["waves"]),
                           "loops_running_max": int(st["loops_running_max"]),
                           "loop_launches": int(st["loop_launches"]), "idle_exits": int(st["idle_exits"]),
                           "device_mb": st["device_bytes"] / 2 ** 20,
                           "arena_peak_mb": st["arena_peak"] / 2 ** 20},
                "plain_per_call": {"p50_ms": 1e3 * _pct(lat_p, 50), "p99_ms": 1e3 * _pct(lat_p, 99),
                                   "solves_s": sets / span_p}})
    top = sweep[-1]
    line = _line(args, top["served"]["solves_s"], None,
                 "c5: 4 resident matrices (Gaussian/Rademacher 1024x4096, Gaussian 2048x16384, correlated "
                 "1024x4096); open-loop Poisson requests, k ~ U[8,512], 1-4096 sets log-uniform; served "
                 "(4 device-resident request loops over one oldest-first table, 2 GiB HBM budget) vs one pl_solve call per request", {
                     "serve": {"capacity_req_s": cap, "capacity_solves_s": cal_sets / cap_s,
                               "plain_capacity_req_s": len(cal) / cap_plain_s,
                               "plain_capacity_solves_s": cal_sets / cap_plain_s,
                               "capacity_note": "the same 40 requests submitted at once (closed burst)",
                               "sweep": sweep,
                               "p50_ms": top["served"]["p50_ms"], "p99_ms": top["served"]["p99_ms"],
                               "plain_p50_ms": top["plain_per_call"]["p50_ms"],
                               "plain_p99_ms": top["plain_per_call"]["p99_ms"]},
                     "e2e": {"value": top["served"]["solves_s"], "unit": "solves/s",
                             "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                             "path": "pl_serve_submit / pl_serve_wait with host buffers (per request)"},
                     "gpu_launches": None})
    line["value_note"] = "solves/s of the server at the highest swept rate (open loop)"
    print(json.dumps(line), flush=True)
    return 0


def run(args):
    if args.impl == "reference":
        print(json.dumps({"impl": "reference", "unavailable": "the CPU reference arm covers the default c2 "
                          "workload only; c1, c3-c5 report their CPU sample under cpu_baseline"}))
        return 0
    return {"c1": run_c1, "c3": run_c3, "c4": run_c4, "c5": run_c5}[args.workload](args)
