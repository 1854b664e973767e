// pl_sturm.cuh -- FP64 Sturm-count bisection on the Lanczos tridiagonal.
//
// Replaces the reference's serial one-lane TQLRAT (ParaLanczos.cu:32-189, called
// at ParaLanczos.cu:1461).  The count of eigenvalues of T below x is the number of
// sign changes of the leading principal minors of T - xI (continuant form,
// division-free, with power-of-two rescaling every 8 rows).  The reference's
// own Sturm sketch, EIGVALS_BELOW (ParaLanczos.cu:519-552), is unused and skips
// alpha[1]; this is new code.  The CPU restatement is orc_sturm_count in
// oracle/pl_oracle.c.
#pragma once
#include <cuda_runtime.h>

namespace pl {

// Power-of-two rescaling of the last two minors, applied when the exponent of
// p1 leaves [2^-200, 2^200]: exact, keeps signs and ratios.
__device__ __forceinline__ void sturm_rescale(double& p0, double& p1) {
  const int e = ((__double2hiint(p1) >> 20) & 0x7ff) - 1022;  // |p1| = f * 2^e, f in [0.5, 1)
  if (e > 200 || e < -200) {
    const int c = e < -1021 ? -1021 : (e > 1021 ? 1021 : e);
    const double s = __hiloint2double((1023 - c) << 20, 0);  // exactly 2^-c
    p0 *= s;
    p1 *= s;
  }
}

// Number of eigenvalues of T strictly below x.  ab[i] = {alpha_i, beta_i^2}
// (beta_0^2 unused), beta_i^2 > 0 for i >= 1 (a decoupled block stores 2^-600,
// so two consecutive minors cannot both vanish).  Sign changes of the leading
// principal minors p_0 = 1, p_i = (alpha_i - x) p_{i-1} - beta_i^2 p_{i-2}; a
// minor that is exactly zero counts as positive, which gives the right count
// because its neighbours then have opposite signs.
__device__ __forceinline__ int sturm_count(const double2* __restrict__ ab, int k, double x) {
  double p0 = 1.0, p1 = ab[0].x - x;
  unsigned sp = (unsigned)__double2hiint(p1) >> 31;
  int cnt = (int)sp;
  int i = 1;
  for (; i + 16 <= k; i += 16) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const double2 t = ab[i + u];
      const double p2 = fma(t.x - x, p1, -t.y * p0);
      const unsigned s2 = (unsigned)__double2hiint(p2) >> 31;
      cnt += (int)(s2 ^ sp);
      sp = s2;
      p0 = p1;
      p1 = p2;
    }
    sturm_rescale(p0, p1);
  }
  for (; i < k; ++i) {
    const double2 t = ab[i];
    const double p2 = fma(t.x - x, p1, -t.y * p0);
    const unsigned s2 = (unsigned)__double2hiint(p2) >> 31;
    cnt += (int)(s2 ^ sp);
    sp = s2;
    p0 = p1;
    p1 = p2;
  }
  return cnt;
}

// Same count over a strided tridiagonal: element i at ab[i * stride].
__device__ __forceinline__ int sturm_count_strided(const double2* __restrict__ ab, int stride, int k,
                                                   double x) {
  double p0 = 1.0, p1 = ab[0].x - x;
  unsigned sp = (unsigned)__double2hiint(p1) >> 31;
  int cnt = (int)sp;
  int i = 1;
  for (; i + 16 <= k; i += 16) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const double2 t = ab[(size_t)(i + u) * stride];
      const double p2 = fma(t.x - x, p1, -t.y * p0);
      const unsigned s2 = (unsigned)__double2hiint(p2) >> 31;
      cnt += (int)(s2 ^ sp);
      sp = s2;
      p0 = p1;
      p1 = p2;
    }
    sturm_rescale(p0, p1);
  }
  for (; i < k; ++i) {
    const double2 t = ab[(size_t)i * stride];
    const double p2 = fma(t.x - x, p1, -t.y * p0);
    const unsigned s2 = (unsigned)__double2hiint(p2) >> 31;
    cnt += (int)(s2 ^ sp);
    sp = s2;
    p0 = p1;
    p1 = p2;
  }
  return cnt;
}

// Termination width for an interval whose ends have magnitude up to `mag`.
// 2^-34 (6e-11) of the spectrum's scale: far below the FP32 Lanczos error.
__device__ __forceinline__ double bisect_tol(double lo, double hi) {
  return 0x1p-34 * fmax(fabs(lo), fabs(hi)) + 1e-300;
}

// Rounds of (G+1)-way multisection needed to shrink [lo, hi] below tol.
__device__ __forceinline__ int multisect_rounds(double lo, double hi, int G) {
  double w = hi - lo, tol = bisect_tol(lo, hi);
  int r = 0;
  while (w > tol && r < 80) {
    w /= (double)(G + 1);
    ++r;
  }
  return r;
}

// lambda_min and lambda_max by (G+1)-way multisection.  Called by the 2G lanes
// [base, base+2G) of one warp (mask covers exactly them): lanes base..base+G-1
// bracket lambda_min, lanes base+G..base+2G-1 bracket lambda_max, each lane
// evaluating one Sturm count per round.  All callers get both results.
__device__ __forceinline__ void multisect_extremes(const double2* __restrict__ ab, int k,
                                                   double lo, double hi, int G, int base,
                                                   unsigned mask, double& lmin, double& lmax) {
  const int lane = (threadIdx.x & 31) - base;
  const bool isMax = lane >= G;
  const int gi = isMax ? lane - G : lane;
  const int target = isMax ? k : 1;
  const unsigned gm = (G >= 32) ? 0xffffffffu : ((1u << G) - 1u);
  const int shift = base + (isMax ? G : 0);
  const int R = multisect_rounds(lo, hi, G);
  double a = lo, b = hi;
  for (int r = 0; r < R; ++r) {
    const double step = (b - a) / (double)(G + 1);
    const double x = a + step * (double)(gi + 1);
    const bool pass = sturm_count(ab, k, x) >= target;
    const unsigned bal = __ballot_sync(mask, pass);
    const unsigned mine = (bal >> shift) & gm;
    const int f = mine ? (__ffs(mine) - 1) : G;  // first sub-lane whose point passed
    const double na = (f > 0) ? a + step * (double)f : a;
    const double nb = (f < G) ? a + step * (double)(f + 1) : b;
    a = na;
    b = nb;
  }
  const double res = 0.5 * (a + b);
  lmin = __shfl_sync(mask, res, base);
  lmax = __shfl_sync(mask, res, base + G);
}

// One extreme by (G+1)-way multisection with the G = 32 lanes of one warp:
// the smallest x with count(x) >= target (target 1: lambda_min; k: lambda_max).
__device__ __forceinline__ double multisect_warp(const double2* __restrict__ ab, int k, double lo,
                                                 double hi, int target) {
  constexpr int G = 32;
  const int gi = threadIdx.x & 31;
  const int R = multisect_rounds(lo, hi, G);
  double a = lo, b = hi;
  for (int r = 0; r < R; ++r) {
    const double step = (b - a) / (double)(G + 1);
    const double x = a + step * (double)(gi + 1);
    const unsigned bal = __ballot_sync(0xffffffffu, sturm_count(ab, k, x) >= target);
    const int f = bal ? (__ffs(bal) - 1) : G;
    const double na = (f > 0) ? a + step * (double)f : a;
    const double nb = (f < G) ? a + step * (double)(f + 1) : b;
    a = na;
    b = nb;
  }
  return 0.5 * (a + b);
}

// Eigenvalue number m (0-based, ascending) by R rounds of plain bisection.
__device__ __forceinline__ double bisect_index(const double2* __restrict__ ab, int k, int m,
                                               double lo, double hi, int R) {
  double a = lo, b = hi;
  for (int r = 0; r < R; ++r) {
    const double x = 0.5 * (a + b);
    if (sturm_count(ab, k, x) >= m + 1) b = x; else a = x;
  }
  return 0.5 * (a + b);
}

}  // namespace pl
