// pl_queue.cuh -- deferred, batched extraction of lambda_min / lambda_max.
//
// Bisection inside the Lanczos group (several lanes per extreme, multisection)
// spends most Sturm counts on points that carry little information.  Instead a
// group queues the tridiagonals T of its last Q = NT/2 sets in a per-group slice
// of a global scratch buffer (L2-resident: Q * KB * 16 bytes per group) and then
// bisects them all at once with one thread per extreme: plain bisection, one
// bit per Sturm count, every lane doing distinct useful work.
//
// Buffer layout of one group: T[i][slot] (double2 {alpha_i, beta_i^2}), so the
// lanes of a warp reading element i of their slots touch contiguous memory.
#pragma once
#include "pl_common.cuh"
#include "pl_sturm.cuh"
#include "pl_engine.cuh"

namespace pl {

struct QueueMeta {
  long long set;
  int k;
  int status;
};

// Bisection of the queued sets: threads t < 2 * nslots, thread t takes slot
// t / 2, extreme t % 2 (0: lambda_min, 1: lambda_max).  Every thread of the
// group must call it (it ends with a group-uniform shuffle pattern only inside
// warps whose lanes all participate).
__device__ __forceinline__ void queue_bisect(const double2* __restrict__ T, int Q, int nslots,
                                             const QueueMeta* __restrict__ meta, int t,
                                             const SetOutputs& out, unsigned mask) {
  const int slot = t >> 1;
  const bool active = slot < nslots;
  double lam = 0.0;
  int k = 0, status = 0;
  long long set = -1;
  if (active) {
    k = meta[slot].k;
    status = meta[slot].status;
    set = meta[slot].set;
    const double2* __restrict__ ab = T + slot;
    if (!(status & SET_NONFINITE)) {
      double lo = 1e300, hi = -1e300;
      double bprev = 0.0;
      for (int i = 0; i < k; ++i) {
        const double2 e = ab[(size_t)i * Q];
        const double bnext = (i + 1 < k) ? sqrt(ab[(size_t)(i + 1) * Q].y) : 0.0;
        const double rad = bprev + bnext;
        lo = fmin(lo, e.x - rad);
        hi = fmax(hi, e.x + rad);
        bprev = bnext;
      }
      const double pad = 0x1p-51 * fmax(fabs(lo), fabs(hi)) + 1e-300;
      double a = lo - pad, b = hi + pad;
      const int target = (t & 1) ? k : 1;
      const double tol = bisect_tol(a, b);
      for (int r = 0; r < 200 && b - a > tol; ++r) {
        const double x = 0.5 * (a + b);
        if (sturm_count_strided(ab, Q, k, x) >= target) b = x; else a = x;
      }
      lam = 0.5 * (a + b);
    }
  }
  // the partner lane holds the other extreme of the same set
  const double other = __shfl_xor_sync(mask, lam, 1);
  if (active && (t & 1) == 0) {
    if (status & SET_NONFINITE) {
      write_failed(out, set, 0, 0, status);
    } else {
      if (out.lmin) out.lmin[set] = lam;
      if (out.lmax) out.lmax[set] = other;
      if (out.delta) out.delta[set] = fmax(1.0 - lam, other - 1.0);
      if (out.err) out.err[set] = status;
    }
  }
}

}  // namespace pl
