"""Counter-based index-set generator, pure-Python twin of csrc/pl_indexgen.cuh.

Set s of stream `seed` depends only on (seed, s): k distinct values in [0, n)
by Floyd's sampling with SplitMix64 draws mapped to [0, j] by the high half of
a 64x64-bit product.  The reference has no generator (its callers hand in
subIndex, ParaLanczos.cu:1843-1845); the bits here are the project's own
definition and match the device and C implementations exactly.
"""
from __future__ import annotations

import hashlib

import numpy as np

M64 = (1 << 64) - 1
KDIST_FIXED, KDIST_INV_K, KDIST_UNIFORM = 0, 1, 2
INV_K_VALUES = (8, 16, 24, 32, 48, 64, 96, 128, 192, 256)
INV_K_CUM = (96, 144, 176, 200, 216, 228, 236, 242, 246, 249)


def splitmix64(x: int) -> int:
    z = (x + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def set_key(seed: int, s: int) -> int:
    return splitmix64((seed * 0x9E3779B97F4A7C15 + s) & M64)


def set_draw(key: int, i: int) -> int:
    return splitmix64(key ^ ((0x632BE59BD9B4E019 * (i + 1)) & M64))


def gen_k(seed: int, s: int, kdist: int = KDIST_FIXED, kmin: int = 16, kmax: int = 16) -> int:
    if kdist == KDIST_FIXED:
        return kmin
    r = set_draw(set_key(seed, s), 0xFFFFFFFF)
    if kdist == KDIST_INV_K:
        u = (r * 249) >> 64
        for kv, c in zip(INV_K_VALUES, INV_K_CUM):
            if u < c:
                return kv
        return 256
    return kmin + ((r * (kmax - kmin + 1)) >> 64)


def gen_set(seed: int, s: int, n: int, k: int) -> list[int]:
    key = set_key(seed, s)
    out: list[int] = []
    for t in range(k):
        j = n - k + t
        v = (set_draw(key, t) * (j + 1)) >> 64
        out.append(j if v in out else v)
    return out


def gen_stream(seed: int, first: int, nsets: int, n: int, kdist: int = KDIST_FIXED,
               kmin: int = 16, kmax: int = 16):
    """(offsets int64[nsets+1], idx int32[total]) for sets first..first+nsets-1."""
    offs = [0]
    idx: list[int] = []
    for s in range(first, first + nsets):
        k = gen_k(seed, s, kdist, kmin, kmax)
        idx.extend(gen_set(seed, s, n, k))
        offs.append(len(idx))
    return np.asarray(offs, dtype=np.int64), np.asarray(idx, dtype=np.int32)


def stream_sha256(offsets, idx) -> str:
    """SHA-256 over little-endian int64 offsets followed by int32 indices."""
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(offsets, dtype="<i8").tobytes())
    h.update(np.ascontiguousarray(idx, dtype="<i4").tobytes())
    return h.hexdigest()
