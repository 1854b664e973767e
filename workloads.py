"""Seeded synthetic inputs of the five benchmark configurations.

Bench- and test-side only (bench.py, bench_extra.py, profile_case.py and
tests/ import it; the library does not).  Every matrix is built on the host
with numpy, so the GPU arm, the CPU reference arm and the parity tests see the
same bits:

  * a frame Phi (m x n) is drawn in FP64 from ``numpy.random.default_rng(seed)``
    (standard normal / sqrt(m), or Rademacher +-1/sqrt(m)) and stored FP32;
  * A = Phi^T Phi is formed in FP64 from the FP32 frame and stored FP32 (the
    FP64 product is what the drop-in path and dsyev see);
  * index sets come from the project's counter-based generator (seed 1), which
    the library (``api.gen_sets`` / ``api.gen_stream_host``) and the oracle
    implement bit-identically.

The reference publishes no dataset; these stand in for its use (random frames
for RIP studies, ParaLanczos.tex:8-37).
"""
from __future__ import annotations

import functools

import numpy as np

SEED_PHI = 0
SEED_SETS = 1

# (m, n, k, nsets) of the configurations with a fixed k
C1 = dict(m=128, n=512, k=16, nsets=10_000)
C2 = dict(m=1024, n=4096, k=64, nsets=1_000_000)
C3 = dict(m=1024, n=4096, nsets=300_000, kvalues=(8, 16, 24, 32, 48, 64, 96, 128, 192, 256))
C4 = dict(m=2048, n=16384, k=128, nsets=500_000)


def frame(m: int, n: int, seed: int = SEED_PHI, kind: str = "gauss") -> np.ndarray:
    """FP32 frame Phi (m x n, row-major): "gauss" N(0, 1/m), "rademacher"
    +-1/sqrt(m), or "corr" = G (I + 0.3 T) with G Gaussian and T the
    tridiagonal of ones without its diagonal (column j of Phi mixes 0.3 of
    columns j-1 and j+1 of G into column j)."""
    rng = np.random.default_rng(seed)
    if kind == "rademacher":
        P = (rng.integers(0, 2, size=(m, n)).astype(np.float64) * 2.0 - 1.0) / np.sqrt(m)
    else:
        P = rng.standard_normal((m, n)) / np.sqrt(m)
        if kind == "corr":
            Q = P.copy()
            Q[:, 1:] += 0.3 * P[:, :-1]
            Q[:, :-1] += 0.3 * P[:, 1:]
            P = Q
    return np.ascontiguousarray(P, dtype=np.float32)


def gram64(Phi: np.ndarray) -> np.ndarray:
    """A = Phi^T Phi in FP64 of the (FP32) frame."""
    P = Phi.astype(np.float64)
    return P.T @ P


@functools.lru_cache(maxsize=4)
def gram_pair(m: int, n: int, seed: int = SEED_PHI, kind: str = "gauss"):
    """(A64, A32) of the frame(m, n, seed, kind); cached per process."""
    A64 = gram64(frame(m, n, seed, kind))
    A64.setflags(write=False)
    A32 = A64.astype(np.float32)
    A32.setflags(write=False)
    return A64, A32


def c1_matrix():
    """C1: Phi 128 x 512 N(0, 1/128), seed 0 -> (A64, A32), 512 x 512."""
    return gram_pair(C1["m"], C1["n"])


def c2_matrix():
    """C2 / C3: Phi 1024 x 4096 N(0, 1/1024), seed 0 -> (A64, A32), 4096 x 4096."""
    return gram_pair(C2["m"], C2["n"])


def c4_frame(kind: str = "gauss") -> np.ndarray:
    """C4: Phi 2048 x 16384 FP32, Gaussian or Rademacher, seed 0."""
    return frame(C4["m"], C4["n"], SEED_PHI, kind)


# C5's four resident matrices: (label, m, n, kind, seed)
C5_MATRICES = (("gauss 1024x4096", 1024, 4096, "gauss", 100),
               ("rademacher 1024x4096", 1024, 4096, "rademacher", 101),
               ("gauss 2048x16384", 2048, 16384, "gauss", 102),
               ("corr 1024x4096", 1024, 4096, "corr", 103))


def c5_matrix(i: int) -> np.ndarray:
    """FP32 A of C5's matrix i (see C5_MATRICES)."""
    _, m, n, kind, seed = C5_MATRICES[i]
    return gram_pair(m, n, seed, kind)[1]
