// pl_engine.cuh -- register-resident per-set Lanczos for sm_100a.
//
// Replaces the hot loop of POS_SYM_SUBMATRIX_KER2 / POS_SYM_SUBMATRIX_KER
// (ParaLanczos.cu:1285-1374 and 963-1050): gather A[S,S], k Lanczos steps,
// eigenvalues of the tridiagonal.  Differences from the reference, by design:
//   * start vector all-ones/sqrt(k) (the reference draws a clock-seeded cuRAND
//     normal vector, ParaLanczos.cu:1196-1233);
//   * FP32 vectors and matvecs with FP32 accumulation, FP64 alpha/beta;
//   * full reorthogonalisation: after the three-term step
//     w~ = A v_j - alpha_j v_j - beta_j v_{j-1}, w = P_j w~ with the explicit
//     projector P_j = I - sum_{i<=j} v_i v_i^T kept next to A in registers and
//     updated by P -= v v^T in the same pass as the next matvec.  No Lanczos
//     basis is stored and no cross-lane reduce-scatter is needed: the only
//     reductions per step are alpha and ||w||^2;
//   * eigenvalues by FP64 Sturm multisection (pl_sturm.cuh) instead of the
//     one-lane TQLRAT;
//   * breakdown (beta below 32 eps32 ||A_S||_F) restarts from the column of P
//     with the largest diagonal, with beta set to 0 (block-diagonal T);
//   * the warp-synchronous shared-memory hand-offs of the reference
//     (ParaLanczos.cu:1331, 1371, 1454-1478) are explicit __syncwarp /
//     named barriers here.
//
// Thread mapping for one set ("group" of NT threads): a thread owns RPT rows
// (rows rs, rs + KB/RPT, ...) and one of TPR column slices of width KB/TPR, for
// both A_S and P.  Rows/cols >= k are zero padding.
#pragma once
#include "pl_common.cuh"
#include "pl_sturm.cuh"

namespace pl {

template <int KB, int RPT, int TPR>
struct Cfg {
  static constexpr int RSLOTS = KB / RPT;           // distinct row slots
  static constexpr int NT = RSLOTS * TPR;           // threads per set
  static constexpr int CPT = KB / TPR;              // columns per thread
  static constexpr int NW = NT > 32 ? NT / 32 : 1;  // warps per set
  static_assert(KB % RPT == 0 && KB % TPR == 0, "bad shape");
  static_assert(NT <= 32 ? (32 % NT == 0) : (NT % 32 == 0), "bad group size");
  static_assert(CPT % 4 == 0, "column slices are read as float4");
  static_assert(TPR == 1 || TPR == 2, "TPR must be 1 or 2");
};

template <int KB, int NW>
struct __align__(16) GroupSmem {
  float vb[KB];         // broadcast of the (unnormalised) next Lanczos vector
  float wb[KB];         // broadcast of the three-term residual w~
  int idx[KB];          // the set's indices
  double2 ab[KB];       // T: ab[i] = {alpha_i, beta_i^2}, beta_i couples rows i-1, i
  double red[6][NW];    // cross-warp partials (slots 4/5: lambda_min/max hand-off)
};

template <int NT>
struct Grp {
  int t;          // thread index within the group
  unsigned mask;  // this group's lanes within its warp
  int wig;        // warp index within the group
  int bar;        // named barrier id (NT > 32)
  __device__ __forceinline__ void sync() const {
    if constexpr (NT <= 32) {
      __syncwarp(mask);
    } else {
      asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(NT) : "memory");
    }
  }
};

template <int NT>
__device__ __forceinline__ Grp<NT> make_group() {
  Grp<NT> g;
  g.t = threadIdx.x % NT;
  const int lane = threadIdx.x & 31;
  if constexpr (NT < 32) {
    g.mask = ((1u << NT) - 1u) << ((lane / NT) * NT);
  } else {
    g.mask = 0xffffffffu;
  }
  g.wig = g.t / 32;
  g.bar = 1 + (int)(threadIdx.x / NT);
  return g;
}

// Sum over the group; identical (bitwise) result in every thread.
template <int NT, int NW>
__device__ __forceinline__ double group_sum(double x, const Grp<NT>& g, double* red) {
  constexpr int W = NT < 32 ? NT : 32;
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) x += __shfl_xor_sync(g.mask, x, o);
  if constexpr (NW == 1) {
    return x;
  } else {
    if ((threadIdx.x & 31) == 0) red[g.wig] = x;
    g.sync();
    double s = red[0];
#pragma unroll
    for (int w = 1; w < NW; ++w) s += red[w];
    return s;
  }
}

template <int NT, int NW, bool IS_MAX>
__device__ __forceinline__ double group_minmax(double x, const Grp<NT>& g, double* red) {
  constexpr int W = NT < 32 ? NT : 32;
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) {
    const double y = __shfl_xor_sync(g.mask, x, o);
    x = IS_MAX ? fmax(x, y) : fmin(x, y);
  }
  if constexpr (NW == 1) {
    return x;
  } else {
    if ((threadIdx.x & 31) == 0) red[g.wig] = x;
    g.sync();
    double s = red[0];
#pragma unroll
    for (int w = 1; w < NW; ++w) s = IS_MAX ? fmax(s, red[w]) : fmin(s, red[w]);
    return s;
  }
}

template <int NT, int NW>
__device__ __forceinline__ bool group_any(bool p, const Grp<NT>& g, double* red) {
  const bool w = __any_sync(g.mask, p);
  if constexpr (NW == 1) {
    return w;
  } else {
    if ((threadIdx.x & 31) == 0) red[g.wig] = w ? 1.0 : 0.0;
    g.sync();
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < NW; ++i) s += red[i];
    return s != 0.0;
  }
}

// Largest key over the group (keys are unique per row).
template <int NT, int NW>
__device__ __forceinline__ unsigned long long group_max_u64(unsigned long long x, const Grp<NT>& g,
                                                            double* red) {
  constexpr int W = NT < 32 ? NT : 32;
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(g.mask, x, o);
    x = y > x ? y : x;
  }
  if constexpr (NW == 1) {
    return x;
  } else {
    if ((threadIdx.x & 31) == 0) red[g.wig] = __longlong_as_double((long long)x);
    g.sync();
    unsigned long long s = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
      const unsigned long long y = (unsigned long long)__double_as_longlong(red[w]);
      s = y > s ? y : s;
    }
    return s;
  }
}

__device__ __forceinline__ void write_failed(const SetOutputs& out, long long set, long long off,
                                             int k, int status) {
  const double nan = __longlong_as_double(0x7ff8000000000000LL);
  if (out.lmin) out.lmin[set] = nan;
  if (out.lmax) out.lmax[set] = nan;
  if (out.delta) out.delta[set] = nan;
  if (out.det) out.det[set] = nan;
  if (out.err) out.err[set] = status;
  if (out.eig && k > 0)
    for (int m = 0; m < k; ++m) out.eig[off + m] = nan;
}

// Solve one set with the calling group.  S: the set's k indices (global).
template <int KB, int RPT, int TPR, bool ALL>
__device__ __forceinline__ int solve_set(const MatrixF32& M, const int* __restrict__ S, int k,
                                          long long set, long long off, const SetOutputs& out,
                                          GroupSmem<KB, Cfg<KB, RPT, TPR>::NW>& sm,
                                          const Grp<Cfg<KB, RPT, TPR>::NT>& g) {
  using C = Cfg<KB, RPT, TPR>;
  constexpr int NT = C::NT;
  constexpr int NW = C::NW;
  constexpr int CPT = C::CPT;
  const int t = g.t;
  const int rs = t / TPR;
  const int c0 = (t % TPR) * CPT;
  const bool lead = (t % TPR) == 0;  // one thread per row contributes to row reductions

  // ---- indices -> shared memory, validation --------------------------------
  const SetMatrix SM = set_matrix(M, set);
  bool bad = false;
  for (int c = t; c < KB; c += NT) {
    int v = 0;
    if (c < k) {
      v = SM.index(S, c);
      bad |= (v < 0) | (v >= SM.n);
    }
    sm.idx[c] = (c < k && v >= 0 && v < SM.n) ? v : 0;
  }
  if (group_any<NT, NW>(bad, g, sm.red[3])) {
    if (t == 0) write_failed(out, set, off, ALL ? k : 0, SET_BAD_INDEX);
    g.sync();
    return -1;
  }
  g.sync();

  // ---- gather A[S,S] rows into registers; P = I ------------------------------
  // rows stored as column pairs: packed FP32 (FFMA2) halves the FMA issues
  float2 Ar[RPT][CPT / 2];
  float2 Pr[RPT][CPT / 2];
  int rowid[RPT];
  double fro = 0.0;
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    const int r = rs + q * C::RSLOTS;
    rowid[q] = r;
    const bool rv = r < k;
    const float* __restrict__ arow = SM.A + (size_t)sm.idx[r] * (size_t)SM.lda;
#pragma unroll
    for (int cc = 0; cc < CPT; cc += 2) {
      const int c = c0 + cc;
      const float a0 = (rv && c < k) ? __ldg(arow + sm.idx[c]) : 0.f;
      const float a1 = (rv && c + 1 < k) ? __ldg(arow + sm.idx[c + 1]) : 0.f;
      Ar[q][cc / 2] = make_float2(a0, a1);
      Pr[q][cc / 2] = make_float2((rv && c == r) ? 1.f : 0.f, (rv && c + 1 == r) ? 1.f : 0.f);
      fro += (double)a0 * (double)a0 + (double)a1 * (double)a1;
    }
  }
  const double fro2 = group_sum<NT, NW>(fro, g, sm.red[2]);
  const double tau = 32.0 * (double)kEps32 * sqrt(fro2);

  // ---- Lanczos with projector reorthogonalisation ----------------------------
  float v[RPT], vp[RPT];
  const float v0 = (float)(1.0 / sqrt((double)k));
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    v[q] = rowid[q] < k ? v0 : 0.f;
    vp[q] = 0.f;
  }
  for (int c = t; c < KB; c += NT) sm.vb[c] = c < k ? v0 : 0.f;
  float sc = 1.f;     // v = sc * vb (vb holds the unnormalised vector)
  float bprev = 0.f;  // beta_j for the three-term step
  int status = 0;
  g.sync();

  for (int j = 0; j < k; ++j) {
    // P -= v v^T and y = A v, one pass over the broadcast vector
    float2 ya[RPT], yb[RPT], ncoef[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      ya[q] = make_float2(0.f, 0.f);
      yb[q] = make_float2(0.f, 0.f);
      const float cq = -v[q] * sc;
      ncoef[q] = make_float2(cq, cq);
    }
#pragma unroll
    for (int cc = 0; cc < CPT; cc += 4) {
      const float4 b4 = *reinterpret_cast<const float4*>(&sm.vb[c0 + cc]);
      const float2 b01 = make_float2(b4.x, b4.y), b23 = make_float2(b4.z, b4.w);
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        Pr[q][cc / 2] = __ffma2_rn(ncoef[q], b01, Pr[q][cc / 2]);
        Pr[q][cc / 2 + 1] = __ffma2_rn(ncoef[q], b23, Pr[q][cc / 2 + 1]);
        ya[q] = __ffma2_rn(Ar[q][cc / 2], b01, ya[q]);
        yb[q] = __ffma2_rn(Ar[q][cc / 2 + 1], b23, yb[q]);
      }
    }
    float y[RPT];
    double ap = 0.0;
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      y[q] = ((ya[q].x + ya[q].y) + (yb[q].x + yb[q].y)) * sc;
      if constexpr (TPR == 2) y[q] += __shfl_xor_sync(g.mask, y[q], 1);
      if (lead) ap += (double)v[q] * (double)y[q];
    }
    const double alpha = group_sum<NT, NW>(ap, g, sm.red[0]);
    const float af = (float)alpha;

    // three-term residual, broadcast
    float wt[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      wt[q] = fmaf(-af, v[q], fmaf(-bprev, vp[q], y[q]));
      if (lead) sm.wb[rowid[q]] = wt[q];
    }
    g.sync();

    // w = P w~
    float2 wa[RPT], wb2[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      wa[q] = make_float2(0.f, 0.f);
      wb2[q] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int cc = 0; cc < CPT; cc += 4) {
      const float4 x4 = *reinterpret_cast<const float4*>(&sm.wb[c0 + cc]);
      const float2 x01 = make_float2(x4.x, x4.y), x23 = make_float2(x4.z, x4.w);
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        wa[q] = __ffma2_rn(Pr[q][cc / 2], x01, wa[q]);
        wb2[q] = __ffma2_rn(Pr[q][cc / 2 + 1], x23, wb2[q]);
      }
    }
    float w[RPT];
    double bp = 0.0;
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      w[q] = (wa[q].x + wa[q].y) + (wb2[q].x + wb2[q].y);
      if constexpr (TPR == 2) w[q] += __shfl_xor_sync(g.mask, w[q], 1);
      if (lead) {
        bp += (double)w[q] * (double)w[q];
        sm.vb[rowid[q]] = w[q];  // published by the barrier in the reduction below
      }
    }
    const double b2v = group_sum<NT, NW>(bp, g, sm.red[1]);
    if constexpr (NW == 1) g.sync();
    if (t == 0) {
      sm.ab[j].x = alpha;
      if (j + 1 < k) sm.ab[j + 1].y = b2v;
    }
    if (!isfinite(alpha) || !isfinite(b2v)) {
      status |= SET_NONFINITE;
      break;
    }
    if (j + 1 == k) break;
#pragma unroll
    for (int q = 0; q < RPT; ++q) vp[q] = v[q];
    if (b2v > tau * tau) {
      const float bf = sqrtf((float)b2v);
      const float inv = 1.0f / bf;
      sc = inv;
      bprev = bf;
#pragma unroll
      for (int q = 0; q < RPT; ++q) v[q] = w[q] * inv;
    } else {
      // Breakdown: the Krylov space is (numerically) invariant.  Restart with
      // the column of P (orthogonal to every v so far) of largest diagonal.
      status |= SET_BREAKDOWN;
      unsigned long long key = 0ull;
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const int r = rowid[q];
        if (r < k && r >= c0 && r < c0 + CPT) {
          float d = 0.f;
#pragma unroll
          for (int cc = 0; cc < CPT; cc += 2) {
            if (c0 + cc == r) d = Pr[q][cc / 2].x;
            if (c0 + cc + 1 == r) d = Pr[q][cc / 2].y;
          }
          d = fmaxf(d, 0.f);
          const unsigned long long kk =
              ((unsigned long long)__float_as_uint(d) << 32) | (unsigned)(0x7fffffff - r);
          key = kk > key ? kk : key;
        }
      }
      key = group_max_u64<NT, NW>(key, g, sm.red[3]);
      const int m = 0x7fffffff - (int)(key & 0xffffffffu);
      g.sync();  // every thread has read the w broadcast before it is overwritten
#pragma unroll
      for (int q = 0; q < RPT; ++q)
        if (rowid[q] == m) {
#pragma unroll
          for (int cc = 0; cc < CPT; cc += 2) {
            sm.vb[c0 + cc] = Pr[q][cc / 2].x;
            sm.vb[c0 + cc + 1] = Pr[q][cc / 2].y;
          }
        }
      g.sync();
      double zp = 0.0;
      float z[RPT];
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        z[q] = sm.vb[rowid[q]];
        if (lead) zp += (double)z[q] * (double)z[q];
      }
      const double zz = group_sum<NT, NW>(zp, g, sm.red[1]);
      if (t == 0) sm.ab[j + 1].y = 0x1p-600;  // decoupled block (see sturm_count)
      const float inv = 1.0f / sqrtf((float)zz);
      sc = inv;
      bprev = 0.f;
#pragma unroll
      for (int q = 0; q < RPT; ++q) v[q] = z[q] * inv;
    }
  }
  g.sync();  // alpha / beta2 visible to every thread

  if constexpr (!ALL) {
    // extremes mode: T stays in sm.ab for the caller's deferred bisection
    return status;
  }
  if (status & SET_NONFINITE) {
    if (t == 0) write_failed(out, set, off, ALL ? k : 0, status);
    g.sync();
    return -1;
  }

  // ---- eigenvalues of T by FP64 Sturm bisection --------------------------------
  double glo = 1e300, ghi = -1e300;
  for (int i = t; i < k; i += NT) {
    const double rad = (i > 0 ? sqrt(sm.ab[i].y) : 0.0) + (i + 1 < k ? sqrt(sm.ab[i + 1].y) : 0.0);
    glo = fmin(glo, sm.ab[i].x - rad);
    ghi = fmax(ghi, sm.ab[i].x + rad);
  }
  glo = group_minmax<NT, NW, false>(glo, g, sm.red[2]);
  ghi = group_minmax<NT, NW, true>(ghi, g, sm.red[3]);
  {
    const double pad = 0x1p-51 * fmax(fabs(glo), fabs(ghi)) + 1e-300;
    glo -= pad;
    ghi += pad;
  }

  {
    int R = 0;
    {
      double wdt = ghi - glo, tol = bisect_tol(glo, ghi);
      while (wdt > tol && R < 200) {
        wdt *= 0.5;
        ++R;
      }
    }
    double prod = 1.0;
    for (int m = t; m < k; m += NT) {
      const double e = bisect_index(sm.ab, k, m, glo, ghi, R);
      if (out.eig) out.eig[off + m] = e;
      prod *= e;
      if (m == 0 && out.lmin) out.lmin[set] = e;
      if (m == k - 1 && out.lmax) out.lmax[set] = e;
      if (m == 0) sm.red[4][0] = e;  // lambda_min for delta (read after the sync below)
      if (m == k - 1) sm.red[5][0] = e;
    }
    // product over the group (fixed butterfly order, deterministic)
    {
      constexpr int W = NT < 32 ? NT : 32;
#pragma unroll
      for (int o = W / 2; o > 0; o >>= 1) prod *= __shfl_xor_sync(g.mask, prod, o);
      if constexpr (NW > 1) {
        if ((threadIdx.x & 31) == 0) sm.red[0][g.wig] = prod;
      }
    }
    g.sync();
    if (t == 0) {
      double det = prod;
      if constexpr (NW > 1) {
        det = sm.red[0][0];
        for (int w2 = 1; w2 < NW; ++w2) det *= sm.red[0][w2];
      }
      const double lmin = sm.red[4][0];
      const double lmax = sm.red[5][0];
      if (out.det) out.det[set] = det;
      if (out.delta) out.delta[set] = fmax(1.0 - lmin, lmax - 1.0);
      if (out.err) out.err[set] = status;
    }
  }
  g.sync();
  return -1;
}

}  // namespace pl
