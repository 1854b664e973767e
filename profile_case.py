"""Small, self-contained cases of the library's kernels for profiling.

Each case builds its inputs on the GPU, runs the kernel once to warm up
(module load, scratch allocation) and then `--launches` more times, so a
profiler can skip the first launch and capture the next ones:

    python profile_case.py --case k64 [--nsets 200000]
    ncu --set full --clock-control none -k regex:k_sa_solve -s 1 -c 1 \\
        python profile_case.py --case k64

Cases:
  k48      batched form, k = 48 (the k <= 48 bin's kernel) on the k64 matrix.
  k64      batched form, k = 64, A = Phi^T Phi (Phi 1024 x 4096 N(0, 1/1024),
           workloads.c2_matrix), sets from the counter-based generator
           (seed 1); the tuned variant.
  plain64  the same sets through the one-set-per-block form.
  k96      batched form, k = 96 (the k <= 96 bin's kernel) on the same matrix.
  k128     batched form, k = 128 on the same matrix.
  k192     batched form, k = 192 (one-SM engine of the cluster kernel).
  k256     batched form, k = 256 (thread-block-cluster engine).
  gram     on-the-fly Gram blocks, Phi 2048 x 16384 N(0, 1/2048), k = 128.
  uneven   binned launch over the uneven-k stream (P(k) ~ 1/k, k <= 256).
  gather   the gather alone (pl_gather_blocks), k = 64 on the k64 matrix,
           default 100,000 sets (A[S,S] blocks written to HBM).
"""
from __future__ import annotations

import argparse
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", required=True,
                    choices=["k48", "k64", "plain64", "k96", "k128", "k192", "k256", "gram", "uneven",
                             "gather"])
    ap.add_argument("--nsets", type=int, default=0)
    ap.add_argument("--launches", type=int, default=2)
    ap.add_argument("--variant", type=int, default=-2,
                    help="kernel variant of the case's k bin (pl_tune_describe); default: the tuned one")
    a = ap.parse_args(argv)
    import numpy as np
    import torch

    import workloads as W
    from paralanczos_b200 import api
    if a.variant >= -1:
        kb = {"k48": 48, "k64": 64, "plain64": 64, "k96": 96, "k128": 128, "k192": 192, "k256": 256, "gram": 128, "uneven": 0,
              "gather": 64}[a.case]
        b = next(i for i in range(api.num_bins()) if api.bin_kmax(i) >= kb) if kb else 0
        api.tune_set(b, a.variant)
        print(f"bin {b}: variant {a.variant} ({api.tune_describe(b, max(a.variant, 0))[1]})")
    dev = torch.device("cuda", 0)
    t0 = time.perf_counter()
    if a.case == "gram":
        n, k = W.C4["n"], W.C4["k"]
        nsets = a.nsets or 8192
        Phi = torch.from_numpy(W.c4_frame("gauss")).to(dev)
        gf = api.GramFrame(Phi)
        idx = api.gen_sets(1, 0, nsets, n, k)
        for _ in range(1 + a.launches):
            gf.blocks(idx, k)
    else:
        n = W.C2["n"]
        A = torch.from_numpy(np.array(W.c2_matrix()[1])).to(dev)
        if a.case == "gather":
            k = 64
            nsets = a.nsets or 100_000
            idx = api.gen_sets(1, 0, nsets, n, k)
            blocks = api.gather_blocks(A, idx, k)
            for _ in range(a.launches):
                api.gather_blocks(A, idx, k, out=blocks)
        elif a.case == "uneven":
            nsets = a.nsets or 100_000
            off_h, idx_h = api.gen_stream_host(1, 0, nsets, n, kdist=1)
            idx = torch.from_numpy(idx_h).to(dev)
            off = torch.from_numpy(off_h).to(dev)
            out = api.solve(A, idx, offsets=off)
            for _ in range(a.launches):
                api.solve(A, idx, offsets=off, out=out)
        else:
            k = {"k48": 48, "k64": 64, "plain64": 64, "k96": 96, "k128": 128, "k192": 192, "k256": 256}[a.case]
            nsets = a.nsets or {48: 300_000, 64: 200_000, 96: 80_000, 128: 40_000, 192: 8_000, 256: 4_000}[k]
            form = "plain" if a.case == "plain64" else "batched"
            idx = api.gen_sets(1, 0, nsets, n, k)
            out = api.solve(A, idx, k=k, form=form)
            for _ in range(a.launches):
                api.solve(A, idx, k=k, form=form, out=out)
    torch.cuda.synchronize()
    print(f"case {a.case}: {nsets} sets, {1 + a.launches} launches, {time.perf_counter() - t0:.2f} s")
    return 0


if __name__ == "__main__":
    sys.exit(main())
