// pl_engine_sa2.cuh -- shared-A per-set Lanczos with two threads per row.
//
// The recurrence of pl_engine_sa.cuh (three-term step, w = P w~ with the
// explicit projector, P -= v v^T fused with the next matvec; FP32 vectors,
// FP64 alpha/beta), for 64 < k <= 128 with a group of NT = 128 threads (four
// warps) per set laid out differently: each thread holds RPT = 2 rows and, of
// each, every TPR = 2nd float4 column chunk (columns 4 (h + 2 ch) .. +3,
// h = t % 2).  The projector takes the same 128 registers per thread as with
// one full row per thread, but every thread reads only its half of the
// broadcast vectors v and w~, so a warp's broadcast loads per step halve
// (the shared-memory loads of the one-row-per-thread shape are two thirds
// A_S, one third broadcasts).  Row sums are finished with one xor-shuffle
// between the two threads of a row.  Extremes only (the all-eigenvalue mode
// uses the other shapes of the bin).
//
// A layout: element (r, c), r = rs + q * NR, chunk cc = c / 4 = h + 2 ch,
// lives at float4 index (q * NCHT + ch) * NT + (rs * 2 + h): a thread's chunks
// are conflict-free LDS.128 at compile-time offsets from one base pointer.
#pragma once
#include "pl_engine_sa.cuh"

namespace pl {

template <int KB>
struct CfgSA2 {
  static constexpr int RPT = 2, TPR = 2;
  static constexpr int NR = KB / RPT;        // row slots
  static constexpr int NT = NR * TPR;        // threads per set
  static constexpr int NCHT = KB / 4 / TPR;  // float4 chunks per thread and row
  static constexpr int NW = NT / 32;
  static_assert(NT % 32 == 0 && KB % (4 * TPR) == 0, "bad shape");
};

template <int KB>
struct __align__(16) SA2Smem {
  float4 A[KB * KB / 4];
  float vb[KB];
  float wb[KB];
  int idx[KB];
  double2 ab[KB];
  double red[6][CfgSA2<KB>::NW];
};

template <int KB>
__device__ __forceinline__ int sa2_at(int r, int c) {
  using C = CfgSA2<KB>;
  const int q = r / C::NR, rs = r % C::NR, cc = c >> 2;
  return (((q * C::NCHT + cc / C::TPR) * C::NT + rs * C::TPR + cc % C::TPR) << 2) + (c & 3);
}

// One set on the group (extremes mode: T is left in sm.ab).  Returns the
// status bits, or -1 if the set failed (its outputs are written).
template <int KB>
__device__ __forceinline__ int solve_set_sa2(const MatrixF32& M, const int* __restrict__ S, int k,
                                              long long set, long long off, const SetOutputs& out,
                                              SA2Smem<KB>& sm, const Grp<CfgSA2<KB>::NT>& g) {
  using C = CfgSA2<KB>;
  constexpr int NT = C::NT, NW = C::NW, NR = C::NR, RPT = C::RPT, TPR = C::TPR, NCHT = C::NCHT;
  const int t = g.t;
  const int rs = t / TPR, h = t % TPR;
  const bool lead = h == 0;  // the thread of a row that contributes its row to sums

  // ---- indices -> shared memory, validation ---------------------------------
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
    if (t == 0) write_failed(out, set, off, 0, SET_BAD_INDEX);
    g.sync();
    return -1;
  }
  g.sync();

  // ---- gather A_S into shared memory ---------------------------------------
  double fro = 0.0;
  float4* __restrict__ my = sm.A + t;  // chunk (q, ch) at my[(q * NCHT + ch) * NT]
  if (SM.local && (k & 3) == 0 && (SM.lda & 3) == 0 &&
      (reinterpret_cast<uintptr_t>(SM.A) & 15) == 0) {
    // a pre-formed block: contiguous rows, read as the owned float4 chunks
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const int r = rs + q * NR;
      const float4* __restrict__ arow = reinterpret_cast<const float4*>(SM.A + (size_t)r * (size_t)SM.lda);
#pragma unroll
      for (int ch = 0; ch < NCHT; ++ch) {
        const int cc = h + TPR * ch;
        const float4 a4 = (r < k && 4 * cc < k) ? __ldg(arow + cc) : make_float4(0.f, 0.f, 0.f, 0.f);
        fro += (double)a4.x * (double)a4.x + (double)a4.y * (double)a4.y +
               (double)a4.z * (double)a4.z + (double)a4.w * (double)a4.w;
        my[(q * NCHT + ch) * NT] = a4;
      }
    }
  } else {
    // the upper triangle only (k(k+1)/2 random elements, each its own L1
    // request), each off-diagonal element stored twice; rows p and KB-1-p
    // form a pair of KB+1 upper elements shared by TPP threads
    constexpr int NP = KB / 2, TPP = NT / NP, PER = (KB + TPP) / TPP;
    static_assert(NP * TPP == NT, "row pairs per group");
    float* __restrict__ Af = reinterpret_cast<float*>(sm.A);
    const int p = t % NP, i0 = (t / NP) * PER;
    const int r0 = p, r1 = KB - 1 - p;
    const float* __restrict__ row0 = SM.A + (size_t)sm.idx[r0] * (size_t)SM.lda;
    const float* __restrict__ row1 = SM.A + (size_t)sm.idx[r1] * (size_t)SM.lda;
#pragma unroll 8
    for (int ii = 0; ii < PER; ++ii) {
      const int i = i0 + ii;
      if (TPP > 1 && i > KB) break;
      const bool first = i < KB - p;
      const int r = first ? r0 : r1;
      const int c = first ? p + i : i - 1;  // c >= r
      const float e = (r < k && c < k) ? __ldg((first ? row0 : row1) + sm.idx[c]) : 0.f;
      const double e2 = (double)e * (double)e;
      fro += (c == r) ? e2 : 2.0 * e2;
      Af[sa2_at<KB>(r, c)] = e;
      if (c != r) Af[sa2_at<KB>(c, r)] = e;
    }
  }
  float2 Pr[RPT][NCHT * 2];  // P's column pairs of the owned chunks
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    const int r = rs + q * NR;
    const bool rv = r < k;
#pragma unroll
    for (int ch = 0; ch < NCHT; ++ch) {
      const int c = 4 * (h + TPR * ch);
      Pr[q][2 * ch] = make_float2((rv && c == r) ? 1.f : 0.f, (rv && c + 1 == r) ? 1.f : 0.f);
      Pr[q][2 * ch + 1] = make_float2((rv && c + 2 == r) ? 1.f : 0.f, (rv && c + 3 == r) ? 1.f : 0.f);
    }
  }
  // threads read chunks that others wrote: the barriers below order them
  const double fro2 = group_sum<NT, NW>(fro, g, sm.red[2]);
  const double tau = 32.0 * (double)kEps32 * sqrt(fro2);

  // ---- Lanczos with projector reorthogonalisation ----------------------------
  float v[RPT], vp[RPT];
  const float v0 = (float)(1.0 / sqrt((double)k));
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    v[q] = (rs + q * NR) < k ? v0 : 0.f;
    vp[q] = 0.f;
  }
  for (int c = t; c < KB; c += NT) sm.vb[c] = c < k ? v0 : 0.f;
  if (t == 0) sm.ab[0].y = 0.0;
  float sc = 1.f, bprev = 0.f;
  int status = 0;
  g.sync();

  for (int j = 0; j < k; ++j) {
    // P -= v v^T and y = A v over the owned chunks
    float2 ya[RPT], yb[RPT], ncoef[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const float cq = -v[q] * sc;
      ncoef[q] = make_float2(cq, cq);
      ya[q] = make_float2(0.f, 0.f);
      yb[q] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int ch = 0; ch < NCHT; ++ch) {
      const float4 b4 = *reinterpret_cast<const float4*>(&sm.vb[4 * (h + TPR * ch)]);
      const float2 b01 = make_float2(b4.x, b4.y), b23 = make_float2(b4.z, b4.w);
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const float4 a4 = my[(q * NCHT + ch) * NT];
        Pr[q][2 * ch] = __ffma2_rn(ncoef[q], b01, Pr[q][2 * ch]);
        Pr[q][2 * ch + 1] = __ffma2_rn(ncoef[q], b23, Pr[q][2 * ch + 1]);
        ya[q] = __ffma2_rn(make_float2(a4.x, a4.y), b01, ya[q]);
        yb[q] = __ffma2_rn(make_float2(a4.z, a4.w), b23, yb[q]);
      }
    }
    float yy[RPT];
    double ap = 0.0;
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const float part = (ya[q].x + ya[q].y) + (yb[q].x + yb[q].y);
      const float other = __shfl_xor_sync(0xffffffffu, part, 1);
      yy[q] = (part + other) * sc;  // the same sum on both threads (addition commutes)
      if (lead) ap = fma((double)v[q], (double)yy[q], ap);
    }
    const double alpha = group_sum<NT, NW>(ap, g, sm.red[0]);
    const float af = (float)alpha;

    float wt[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      wt[q] = fmaf(-af, v[q], fmaf(-bprev, vp[q], yy[q]));
      if (lead) sm.wb[rs + q * NR] = wt[q];
    }
    g.sync();

    // w = P w~ over the owned chunks
    float2 wa[RPT], wc[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      wa[q] = make_float2(0.f, 0.f);
      wc[q] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int ch = 0; ch < NCHT; ++ch) {
      const float4 x4 = *reinterpret_cast<const float4*>(&sm.wb[4 * (h + TPR * ch)]);
      const float2 x01 = make_float2(x4.x, x4.y), x23 = make_float2(x4.z, x4.w);
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        wa[q] = __ffma2_rn(Pr[q][2 * ch], x01, wa[q]);
        wc[q] = __ffma2_rn(Pr[q][2 * ch + 1], x23, wc[q]);
      }
    }
    float ww[RPT];
    double bp = 0.0;
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const float part = (wa[q].x + wa[q].y) + (wc[q].x + wc[q].y);
      const float other = __shfl_xor_sync(0xffffffffu, part, 1);
      ww[q] = part + other;
      if (lead) {
        bp = fma((double)ww[q], (double)ww[q], bp);
        sm.vb[rs + q * NR] = ww[q];  // published by the barrier inside group_sum
      }
    }
    const double b2v = group_sum<NT, NW>(bp, g, sm.red[1]);
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
      for (int q = 0; q < RPT; ++q) v[q] = ww[q] * inv;
    } else {
      // Breakdown: restart with the column of P (orthogonal to every v so
      // far) of largest diagonal; beta_{j+1} = 0 (decoupled block).
      status |= SET_BREAKDOWN;
      unsigned long long key = 0ull;
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const int r = rs + q * NR;
        if (r < k) {
          bool mine = false;
          float d = 0.f;
#pragma unroll
          for (int ch = 0; ch < NCHT; ++ch) {
            const int c = 4 * (h + TPR * ch);
            if (c == r) { d = Pr[q][2 * ch].x; mine = true; }
            if (c + 1 == r) { d = Pr[q][2 * ch].y; mine = true; }
            if (c + 2 == r) { d = Pr[q][2 * ch + 1].x; mine = true; }
            if (c + 3 == r) { d = Pr[q][2 * ch + 1].y; mine = true; }
          }
          if (mine) {
            d = fmaxf(d, 0.f);
            const unsigned long long kk =
                ((unsigned long long)__float_as_uint(d) << 32) | (unsigned)(0x7fffffff - r);
            key = kk > key ? kk : key;
          }
        }
      }
      key = group_max_u64<NT, NW>(key, g, sm.red[3]);
      const int m = 0x7fffffff - (int)(key & 0xffffffffu);
      g.sync();
#pragma unroll
      for (int q = 0; q < RPT; ++q)
        if (rs + q * NR == m) {  // both threads of row m write their chunks of P's row m
#pragma unroll
          for (int ch = 0; ch < NCHT; ++ch) {
            const int c = 4 * (h + TPR * ch);
            sm.vb[c] = Pr[q][2 * ch].x;
            sm.vb[c + 1] = Pr[q][2 * ch].y;
            sm.vb[c + 2] = Pr[q][2 * ch + 1].x;
            sm.vb[c + 3] = Pr[q][2 * ch + 1].y;
          }
        }
      g.sync();
      double zp = 0.0;
      float z[RPT];
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        z[q] = sm.vb[rs + q * NR];
        if (lead) zp += (double)z[q] * (double)z[q];
      }
      const double zz = group_sum<NT, NW>(zp, g, sm.red[4]);
      if (t == 0) sm.ab[j + 1].y = 0x1p-600;  // decoupled block (see sturm_count)
      const float inv = 1.0f / sqrtf((float)zz);
      sc = inv;
      bprev = 0.f;
#pragma unroll
      for (int q = 0; q < RPT; ++q) v[q] = z[q] * inv;
    }
  }
  g.sync();  // T visible to every thread
  return status;
}

}  // namespace pl
