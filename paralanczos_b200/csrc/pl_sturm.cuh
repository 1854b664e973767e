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

__device__ __forceinline__ void sturm_rescale(double& p0, double& p1) {
  double m = fmax(fabs(p0), fabs(p1));
  if (m > 0x1p200 || m < 0x1p-200) {
    int e = ((__double2hiint(m) >> 20) & 0x7ff) - 1022;  // m = f * 2^e, f in [0.5, 1)
    e = e < -1021 ? -1021 : (e > 1021 ? 1021 : e);
    double s = __hiloint2double((1023 - e) << 20, 0);     // exactly 2^-e
    p0 *= s;
    p1 *= s;
  }
}

// Number of eigenvalues of T strictly below x.  al[0..k-1] diagonal,
// b2[i] = beta_i^2 couples rows i-1 and i (b2[0] unused).  A zero minor is
// replaced by a tiny negative one (the pivmin convention), so a count is always
// defined.
__device__ __forceinline__ int sturm_count(const double* __restrict__ al,
                                           const double* __restrict__ b2, int k, double x) {
  double p0 = 1.0, p1 = al[0] - x;
  if (p1 == 0.0) p1 = -0x1p-900;
  bool neg = p1 < 0.0;
  int cnt = neg;
  for (int i = 1; i < k; ++i) {
    double p2 = fma(al[i] - x, p1, -b2[i] * p0);
    if (p2 == 0.0) {
      p2 = -0x1p-900 * fabs(p1);
      if (p2 == 0.0) p2 = -0x1p-1000;
    }
    bool n2 = p2 < 0.0;
    cnt += (n2 != neg);
    neg = n2;
    p0 = p1;
    p1 = p2;
    if ((i & 7) == 7) sturm_rescale(p0, p1);
  }
  return cnt;
}

// Termination width for an interval whose ends have magnitude up to `mag`.
__device__ __forceinline__ double bisect_tol(double lo, double hi) {
  return 0x1p-48 * fmax(fabs(lo), fabs(hi)) + 1e-300;
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
__device__ __forceinline__ void multisect_extremes(const double* __restrict__ al,
                                                   const double* __restrict__ b2, int k,
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
    const bool pass = sturm_count(al, b2, k, x) >= target;
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

// Eigenvalue number m (0-based, ascending) by R rounds of plain bisection.
__device__ __forceinline__ double bisect_index(const double* __restrict__ al,
                                               const double* __restrict__ b2, int k, int m,
                                               double lo, double hi, int R) {
  double a = lo, b = hi;
  for (int r = 0; r < R; ++r) {
    const double x = 0.5 * (a + b);
    if (sturm_count(al, b2, k, x) >= m + 1) b = x; else a = x;
  }
  return 0.5 * (a + b);
}

}  // namespace pl
