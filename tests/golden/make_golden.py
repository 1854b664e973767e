"""Generate the committed golden fixtures under tests/golden/.

    python tests/golden/make_golden.py

Needs the reference tree (for oracle/_ref, the reference's own TQLRAT and
DET_TRIDIAG compiled from its source by oracle/build_ref.py) and scipy.  The
GPU box has no reference tree, so everything the tests need from the reference
is frozen here:

  tqlrat_ref.npz   random and edge-case tridiagonals with the outputs of the
                   reference's compiled TQLRAT/DET_TRIDIAG (pins the oracle's
                   restatement bit-for-bit);
  fixture8.json    the reference's 8x8 SPD test matrix (example1.cu:19-26,
                   Matlab/for_example_3.m:3-10) with the subsets the examples use
                   (example1.cu:39-42, example3.cu:43-49) and the oracle / FP64
                   dsyev answers;
  oracle_sets.npz  submatrices A[S,S] of seeded Gaussian Gram matrices at
                   k = 16, 64, 128: oracle (reference path restated) and dsyev
                   eigenvalues;
  indexgen.json    SHA-256 of generator streams (fixed k, 1/k mix, uniform k).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from paralanczos_b200 import indexgen as IG  # noqa: E402

FIXTURE8 = [
    11.6150, 12.6022, 2.7449, 0.6018, 5.7419, -0.8989, 6.2368, 1.4880,
    12.6022, 32.5907, 6.8222, 3.8457, 3.8868, -1.3879, 7.2553, 1.3472,
    2.7449, 6.8222, 11.3095, 1.9900, -3.8608, 0.9067, 3.4324, 3.3344,
    0.6018, 3.8457, 1.9900, 4.7412, -0.0663, -1.2597, -0.2133, -1.6123,
    5.7419, 3.8868, -3.8608, -0.0663, 18.0182, -1.7439, -1.5991, 1.2881,
    -0.8989, -1.3879, 0.9067, -1.2597, -1.7439, 1.4386, 1.4156, 1.8073,
    6.2368, 7.2553, 3.4324, -0.2133, -1.5991, 1.4156, 8.2406, 2.8208,
    1.4880, 1.3472, 3.3344, -1.6123, 1.2881, 1.8073, 2.8208, 4.7334,
]


def tqlrat_cases():
    rng = np.random.default_rng(20260101)
    cases = []
    for n in [1, 2, 3, 4, 8, 16, 31, 64, 128]:
        for scale in (1e-3, 1.0, 1e3):
            d = rng.standard_normal(n) * scale
            e2 = (rng.standard_normal(n) * scale) ** 2
            cases.append((d, e2))
    # edge cases: zero couplings, repeated diagonals, zero matrix, graded
    cases.append((np.ones(8), np.zeros(8)))
    cases.append((np.zeros(6), np.zeros(6)))
    cases.append((np.array([1.0, 1, 1, 1, 2, 2, 2, 2]), np.full(8, 1e-20)))
    cases.append((np.arange(1, 17, dtype=float), np.r_[0.0, np.full(15, 1.0)]))
    cases.append((np.logspace(-8, 8, 24), np.r_[0.0, np.logspace(-6, 6, 23)]))
    return cases


def main() -> int:
    if O.ref_lib() is None:
        O.build()
    if O.ref_lib() is None:
        print("oracle/_ref is missing: the reference tree is needed to regenerate")
        return 1
    # 1. TQLRAT / DET_TRIDIAG of the reference itself
    ds, e2s, outd, oute2, ierr, dets, lens = [], [], [], [], [], [], []
    for d, e2 in tqlrat_cases():
        dd, ee, ie = O.tqlrat(d, e2, impl="reference")
        det = O.det_tridiag(dd, ee, impl="reference")
        ds.append(d)
        e2s.append(e2)
        outd.append(dd)
        oute2.append(ee)
        ierr.append(ie)
        dets.append(det)
        lens.append(len(d))
    np.savez_compressed(os.path.join(HERE, "tqlrat_ref.npz"), lens=np.array(lens),
                        d=np.concatenate(ds), e2=np.concatenate(e2s), out_d=np.concatenate(outd),
                        out_e2=np.concatenate(oute2), ierr=np.array(ierr), det=np.array(dets))

    # 2. the reference's 8x8 fixture
    g = np.array(FIXTURE8).reshape(8, 8)
    fx = {"matrix": FIXTURE8, "cases": []}
    for S in ([1, 3, 5, 7], list(range(8)), [0, 1, 2, 3], [4, 5, 6, 7]):
        eig, det, ie = O.subset_solve(g, S)
        fx["cases"].append({"subset": S, "oracle_eigs": eig.tolist(), "oracle_det": det, "ierr": ie,
                            "dsyev_eigs": O.dsyev_eigs(g[np.ix_(S, S)]).tolist()})
    with open(os.path.join(HERE, "fixture8.json"), "w") as f:
        json.dump(fx, f, indent=1)

    # 3. seeded Gram matrices: gathered submatrices A[S,S] (float32) of sets from
    #    the project's generator, with the oracle's and dsyev's eigenvalues
    out = {}
    rng = np.random.default_rng(0)
    for (M, N, k, nsets) in [(128, 512, 16, 32), (1024, 4096, 64, 8), (2048, 4096, 128, 2)]:
        Phi = (rng.standard_normal((M, N)) / np.sqrt(M)).astype(np.float32)
        offs, idx = IG.gen_stream(7, 0, nsets, N, 0, k, k)
        sub = []
        for s in range(nsets):
            S = idx[s * k:(s + 1) * k]
            P = Phi[:, S].astype(np.float64)
            sub.append((P.T @ P).astype(np.float32))
        sub = np.stack(sub)
        eigs, dets, ierrs, truth = [], [], [], []
        for s in range(nsets):
            e, d, ie = O.subset_solve(sub[s], np.arange(k, dtype=np.int32))
            eigs.append(e)
            dets.append(d)
            ierrs.append(ie)
            truth.append(O.dsyev_eigs(sub[s]))
        tag = f"M{M}_k{k}"
        out[tag + "_sub"] = sub
        out[tag + "_idx"] = idx
        out[tag + "_oracle_eig"] = np.stack(eigs)
        out[tag + "_oracle_det"] = np.array(dets)
        out[tag + "_oracle_ierr"] = np.array(ierrs)
        out[tag + "_dsyev_eig"] = np.stack(truth)
    np.savez_compressed(os.path.join(HERE, "oracle_sets.npz"), **out)

    # 4. generator streams
    gen = {}
    for name, args in {
        "fixed_n512_k16": (1, 0, 10000, 512, 0, 16, 16),
        "invk_n4096": (3, 0, 3000, 4096, 1, 8, 256),
        "uniform_n4096_8_512": (5, 0, 500, 4096, 2, 8, 512),
        "fixed_n4096_k64_offset": (1, 123456789, 1000, 4096, 0, 64, 64),
    }.items():
        o, i = IG.gen_stream(*args)
        gen[name] = {"args": list(args), "sha256": IG.stream_sha256(o, i), "total": int(o[-1]),
                     "first_set": i[:o[1]].tolist()}
    with open(os.path.join(HERE, "indexgen.json"), "w") as f:
        json.dump(gen, f, indent=1)
    print("golden fixtures written to", HERE)
    return 0


if __name__ == "__main__":
    sys.exit(main())
