// pl_indexgen.cuh -- counter-based index-set generator (host and device).
//
// The reference has no generator: its callers pass subIndex in
// (ParaLanczos.cu:1843-1845, example2.cu:42-48, gpu_multi_subsvd2.m:57).  Set s
// of stream `seed` depends only on (seed, s), so a sweep can be split or
// resumed by set range.  k distinct values in [0, n) by Floyd's sampling with
// SplitMix64 draws mapped to [0, j] by a 64x64->128 high multiply.  The CPU
// oracle (orc_gen_* in oracle/pl_oracle.c) and paralanczos_b200/indexgen.py
// produce the same bits.
#pragma once
#include <stdint.h>
#ifndef PL_HD
#ifdef __CUDACC__
#define PL_HD __host__ __device__ __forceinline__
#else
#define PL_HD inline
#endif
#endif

namespace pl {

PL_HD uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

PL_HD uint64_t set_key(uint64_t seed, uint64_t s) { return splitmix64(seed * 0x9E3779B97F4A7C15ULL + s); }

PL_HD uint64_t set_draw(uint64_t key, uint64_t i) {
  return splitmix64(key ^ (0x632BE59BD9B4E019ULL * (i + 1)));
}

PL_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * (unsigned __int128)b) >> 64);
#endif
}

// k distributions: 0 fixed (kmin); 1 {8,16,24,32,48,64,96,128,192,256} with
// P proportional to 1/k (integer weights 96,48,32,24,16,12,8,6,4,3 of 249);
// 2 uniform in [kmin, kmax].
PL_HD int gen_k(uint64_t seed, uint64_t s, int kdist, int kmin, int kmax) {
  if (kdist == 0) return kmin;
  const uint64_t r = set_draw(set_key(seed, s), 0xFFFFFFFFULL);
  if (kdist == 1) {
    const int kv[10] = {8, 16, 24, 32, 48, 64, 96, 128, 192, 256};
    const int cum[10] = {96, 144, 176, 200, 216, 228, 236, 242, 246, 249};
    const uint64_t u = mulhi64(r, 249);
    for (int i = 0; i < 10; ++i)
      if (u < (uint64_t)cum[i]) return kv[i];
    return 256;
  }
  return kmin + (int)mulhi64(r, (uint64_t)(kmax - kmin + 1));
}

PL_HD void gen_set(uint64_t seed, uint64_t s, int n, int k, int* out) {
  const uint64_t key = set_key(seed, s);
  for (int t = 0; t < k; ++t) {
    const uint64_t j = (uint64_t)(n - k + t);
    const uint64_t v = mulhi64(set_draw(key, (uint64_t)t), j + 1);
    bool dup = false;
    for (int q = 0; q < t; ++q)
      if ((uint64_t)out[q] == v) {
        dup = true;
        break;
      }
    out[t] = dup ? (int)j : (int)v;
  }
}

}  // namespace pl
