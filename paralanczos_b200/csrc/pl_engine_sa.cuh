// pl_engine_sa.cuh -- "shared-A" per-set Lanczos: the projector P in
// registers, A[S,S] in shared memory.
//
// Same recurrence as pl_engine.cuh (three-term step, then w = P w~ with the
// explicit projector P = I - sum v v^T, P -= v v^T fused with the next matvec;
// FP32 vectors, FP64 alpha/beta, FP64 Sturm multisection), but A_S is read
// from shared memory instead of being held in registers.  That halves the
// registers per set, so a k <= 64 set fits one warp (no named barriers, only
// warp shuffles) and twice as many sets are in flight per SM, which is what
// the latency-bound per-step chain y -> alpha -> w~ -> P w~ -> beta needs.
//
// A layout: thread t of a group of NT owns rows r_q = t + q*NT (q < RPT); its
// row data is stored lane-interleaved, A[q][chunk][t][4] (4 floats per chunk),
// so every thread's LDS.128 of its own row chunk is conflict-free and uses a
// compile-time offset from one per-thread base pointer.
#pragma once
#include "pl_engine.cuh"

namespace pl {

template <int KB, int RPT>
struct CfgSA {
  static constexpr int NT = KB / RPT;  // threads per set
  static constexpr int NCH = KB / 4;   // float4 chunks per row
  static constexpr int NW = NT > 32 ? NT / 32 : 1;
  static_assert(KB % RPT == 0 && KB % 4 == 0, "bad shape");
  static_assert(NT <= 32 ? (32 % NT == 0) : (NT % 32 == 0), "bad group size");
};

template <int KB, int RPT>
struct __align__(16) SASmem {
  float4 A[RPT * (KB / 4) * (KB / RPT)];  // [q][chunk][thread] float4
  float vb[KB];
  float wb[KB];
  int idx[KB];
  double2 ab[KB];
  double red[6][CfgSA<KB, RPT>::NW];
};

// Float offset of A_S element (r, c) in the lane-interleaved layout (row
// r = t + q * NT, column c = 4 * ch + u at ((q * NCH + ch) * NT + t) * 4 + u).
template <int NT, int NCH>
__device__ __forceinline__ int sa_at(int r, int c) {
  return (((r / NT) * NCH + (c >> 2)) * NT + (r % NT)) * 4 + (c & 3);
}

// Prefetch of the next set's upper triangle (the PF variants).  While a group
// runs its set's Lanczos steps, its threads issue cp.async copies of the next
// set's k(k+1)/2 random elements of A into a shared-memory stage, a few per
// step; they need no registers and land long before the set ends.  The next
// set then mirrors the stage into its A_S layout instead of gathering from
// global memory.  Thread t stages exactly the elements it would have
// gathered, at e[ii * NT + t] (its ii-th), so it reads back only its own
// copies.
struct SANext {
  SetMatrix SM;
  const int* S;
  int k;
  bool valid;
};

template <int KB, int NT>
struct __align__(16) SAStage {
  // (groups of fewer than KB / 2 threads never prefetch; TPP = 1 keeps the
  // type complete for them)
  static constexpr int NP = KB / 2, TPP = NT >= NP ? NT / NP : 1, PER = (KB + TPP) / TPP;
  float e[PER * NT];
  int idx[KB];  // the next set's indices, -1 outside [0, n)
};

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// The issuing side of the prefetch for one thread: the triangle order of the
// gather (rows p and KB-1-p paired, TPP threads per pair), PKS elements per
// Lanczos step.
template <int KB, int NT>
struct TriPrefetch {
  static constexpr int NP = KB / 2, TPP = NT / NP, PER = (KB + TPP) / TPP;
  static constexpr int PKS = (PER + 31) / 32;
  static_assert(NP * TPP == NT, "row pairs per group");
  const float* row0 = nullptr;
  const float* row1 = nullptr;
  int k = 0, pf = 0;
  bool on = false;

  // the next set's indices into stg->idx (checked), its two row pointers
  template <class G>
  __device__ __forceinline__ void setup(const SANext* nx, SAStage<KB, NT>* stg, const G& g) {
    const int t = g.t, p = t % NP;
    g.sync();  // the previous prefetch's readers of stg->idx are done
    for (int c = t; c < KB; c += NT) {
      int v = -1;
      if (c < nx->k) {
        v = nx->SM.index(nx->S, c);
        if (v < 0 || v >= nx->SM.n) v = -1;
      }
      stg->idx[c] = v;
    }
    g.sync();
    const int a0 = stg->idx[p], a1 = stg->idx[KB - 1 - p];
    row0 = a0 >= 0 ? nx->SM.A + (size_t)a0 * (size_t)nx->SM.lda : nullptr;
    row1 = a1 >= 0 ? nx->SM.A + (size_t)a1 * (size_t)nx->SM.lda : nullptr;
    k = nx->k;
    pf = 0;
    on = true;
  }
  __device__ __forceinline__ void issue(SAStage<KB, NT>* stg, int t, int ii) const {
    const int p = t % NP, i = (t / NP) * PER + ii;
    if (TPP > 1 && i > KB) return;
    const bool first = i < KB - p;
    const int r = first ? p : KB - 1 - p;
    const int c = first ? p + i : i - 1;
    if (r < k && c < k) {
      const int ci = stg->idx[c];
      const float* row = first ? row0 : row1;
      if (row && ci >= 0) cp_async4(&stg->e[ii * NT + t], row + ci);
    }
  }
  __device__ __forceinline__ void step(SAStage<KB, NT>* stg, int t) {
    if (on)
      for (int q = 0; q < PKS && pf < PER; ++q, ++pf) issue(stg, t, pf);
  }
  __device__ __forceinline__ void finish(SAStage<KB, NT>* stg, int t) {
    if (on)
      for (; pf < PER; ++pf) issue(stg, t, pf);
  }
};

template <int KB, int RPT, bool ALL, bool PF = false, int AR = 0>
__device__ __forceinline__ int solve_set_sa(const MatrixF32& M, const int* __restrict__ S, int k,
                                             long long set, long long off, const SetOutputs& out,
                                             SASmem<KB, RPT>& sm,
                                             const Grp<CfgSA<KB, RPT>::NT>& g,
                                             SAStage<KB, KB / RPT>* stg = nullptr, bool have = false,
                                             const SANext* nx = nullptr, bool* issued = nullptr) {
  using C = CfgSA<KB, RPT>;
  constexpr int NT = C::NT;
  constexpr int NW = C::NW;
  constexpr int NCH = C::NCH;
  const int t = g.t;
  if constexpr (PF) {
    static_assert(RPT <= 2 && !ALL, "the prefetch follows the triangle gather (extremes mode)");
    *issued = false;
    if (have) cp_async_wait_all();  // this set's stage (issued a whole set ago)
  }

  // ---- indices -> shared memory, validation ---------------------------------
  // (a prefetched set's indices were read and checked by the previous set:
  // stg->idx, -1 where outside [0, n))
  const SetMatrix SM = set_matrix(M, set);
  bool bad = false;
  for (int c = t; c < KB; c += NT) {
    int v = 0;
    if (c < k) {
      if (PF && have)
        v = stg->idx[c];
      else
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

  // ---- gather this thread's rows of A[S,S] into shared memory; P = I ----------
  float4* __restrict__ my = sm.A + t;  // chunk (q, ch) at my[(q * NCH + ch) * NT]
  float2 Pr[RPT][KB / 2];  // column pairs: packed FP32 (FFMA2) halves the FMA issues
  double fro = 0.0;
  // A pre-formed block (the Gram form) has contiguous rows: with k % 4 == 0 and
  // a 16-byte aligned block they are read as float4 (a quarter of the loads,
  // whose latency is HBM's there).
  const bool vec = SM.local && (k & 3) == 0 && (SM.lda & 3) == 0 &&
                   ((reinterpret_cast<uintptr_t>(SM.A) & 15) == 0);
  bool gathered = false;
  if constexpr (RPT <= 2) {
    if (!vec) {
      // A_S is symmetric: load only its upper triangle, k(k+1)/2 of the k^2
      // random elements (each a separate L1 request and 32-byte sector, the
      // gather's cost), and store each off-diagonal element twice.  Rows p and
      // KB-1-p form a pair with KB+1 upper elements; TPP = 2 / RPT threads
      // share a pair, so every thread loads about the same number.
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
        float e = 0.f;
        if (r < k && c < k) {
          if (PF && have)
            e = stg->e[ii * NT + t];
          else
            e = __ldg((first ? row0 : row1) + sm.idx[c]);
        }
        const double e2 = (double)e * (double)e;
        fro += (c == r) ? e2 : 2.0 * e2;
        Af[sa_at<NT, NCH>(r, c)] = e;
        if (c != r) Af[sa_at<NT, NCH>(c, r)] = e;
      }
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const int r = t + q * NT;
        const bool rv = r < k;
#pragma unroll
        for (int ch = 0; ch < NCH; ++ch) {
          Pr[q][2 * ch] =
              make_float2((rv && 4 * ch == r) ? 1.f : 0.f, (rv && 4 * ch + 1 == r) ? 1.f : 0.f);
          Pr[q][2 * ch + 1] =
              make_float2((rv && 4 * ch + 2 == r) ? 1.f : 0.f, (rv && 4 * ch + 3 == r) ? 1.f : 0.f);
        }
      }
      gathered = true;
    }
  }
  if (!gathered) {
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const int r = t + q * NT;
      const bool rv = r < k;
      const float* __restrict__ arow = SM.A + (size_t)sm.idx[r] * (size_t)SM.lda;
#pragma unroll
      for (int ch = 0; ch < NCH; ++ch) {
        float e[4];
        if (vec) {
          const float4 a4 = (rv && 4 * ch < k) ? __ldg(reinterpret_cast<const float4*>(arow) + ch)
                                               : make_float4(0.f, 0.f, 0.f, 0.f);
          e[0] = a4.x;
          e[1] = a4.y;
          e[2] = a4.z;
          e[3] = a4.w;
        } else {
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int c = 4 * ch + u;
            e[u] = (rv && c < k) ? __ldg(arow + sm.idx[c]) : 0.f;
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) fro += (double)e[u] * (double)e[u];
        Pr[q][2 * ch] = make_float2((rv && 4 * ch == r) ? 1.f : 0.f, (rv && 4 * ch + 1 == r) ? 1.f : 0.f);
        Pr[q][2 * ch + 1] =
            make_float2((rv && 4 * ch + 2 == r) ? 1.f : 0.f, (rv && 4 * ch + 3 == r) ? 1.f : 0.f);
        my[(q * NCH + ch) * NT] = make_float4(e[0], e[1], e[2], e[3]);
      }
    }
  }
  const double fro2 = group_sum<NT, NW>(fro, g, sm.red[2]);
  const double tau = 32.0 * (double)kEps32 * sqrt(fro2);

  // ---- the next set's prefetch: its indices, then its elements over the steps -
  TriPrefetch<KB, PF ? NT : KB> pre;  // (a valid shape when unused)
  if constexpr (PF) {
    if (nx->valid) pre.setup(nx, stg, g);
  }

  // ---- Lanczos with projector reorthogonalisation ----------------------------
  float v[RPT], vp[RPT];
  const float v0 = (float)(1.0 / sqrt((double)k));
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    v[q] = (t + q * NT) < k ? v0 : 0.f;
    vp[q] = 0.f;
  }
  for (int c = t; c < KB; c += NT) sm.vb[c] = c < k ? v0 : 0.f;
  if (t == 0) sm.ab[0].y = 0.0;
  float sc = 1.f, bprev = 0.f;
  int status = 0;
  g.sync();
  // The first AR float4 chunks of each of the thread's rows of A_S are held in
  // registers for the whole recurrence: AR * RPT fewer shared-memory loads per
  // step (the L1 data pipe is the kernel's busiest unit), same products.
  static_assert(AR >= 0 && AR <= NCH, "register chunks of a row");
  float4 Ar[RPT][AR > 0 ? AR : 1];
#pragma unroll
  for (int q = 0; q < RPT; ++q)
#pragma unroll
    for (int ch = 0; ch < AR; ++ch) Ar[q][ch] = my[(q * NCH + ch) * NT];

  for (int j = 0; j < k; ++j) {
    if constexpr (PF) pre.step(stg, t);
    // P -= v v^T and y = A v, one pass over the broadcast vector
    float2 ya[RPT], yb[RPT], ncoef[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const float cq = -v[q] * sc;
      ncoef[q] = make_float2(cq, cq);
      ya[q] = make_float2(0.f, 0.f);
      yb[q] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int ch = 0; ch < NCH; ++ch) {
      const float4 b4 = *reinterpret_cast<const float4*>(&sm.vb[4 * ch]);
      const float2 b01 = make_float2(b4.x, b4.y), b23 = make_float2(b4.z, b4.w);
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const float4 a4 = ch < AR ? Ar[q][ch < AR ? ch : 0] : my[(q * NCH + ch) * NT];
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
      yy[q] = ((ya[q].x + ya[q].y) + (yb[q].x + yb[q].y)) * sc;
      ap = fma((double)v[q], (double)yy[q], ap);
    }
    const double alpha = group_sum<NT, NW>(ap, g, sm.red[0]);
    const float af = (float)alpha;

    float wt[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      wt[q] = fmaf(-af, v[q], fmaf(-bprev, vp[q], yy[q]));
      sm.wb[t + q * NT] = wt[q];
    }
    g.sync();

    // w = P w~
    float2 wa[RPT], wc[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      wa[q] = make_float2(0.f, 0.f);
      wc[q] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int ch = 0; ch < NCH; ++ch) {
      const float4 x4 = *reinterpret_cast<const float4*>(&sm.wb[4 * ch]);
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
      ww[q] = (wa[q].x + wa[q].y) + (wc[q].x + wc[q].y);
      bp = fma((double)ww[q], (double)ww[q], bp);
      sm.vb[t + q * NT] = ww[q];  // published by the sync below
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
      for (int q = 0; q < RPT; ++q) v[q] = ww[q] * inv;
    } else {
      // Breakdown: restart with the column of P (orthogonal to every v so
      // far) of largest diagonal; beta_{j+1} = 0 (decoupled block).
      status |= SET_BREAKDOWN;
      unsigned long long key = 0ull;
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const int r = t + q * NT;
        if (r < k) {
          float d = 0.f;
#pragma unroll
          for (int c = 0; c < KB; c += 2) {
            if (c == r) d = Pr[q][c / 2].x;
            if (c + 1 == r) d = Pr[q][c / 2].y;
          }
          d = fmaxf(d, 0.f);
          const unsigned long long kk =
              ((unsigned long long)__float_as_uint(d) << 32) | (unsigned)(0x7fffffff - r);
          key = kk > key ? kk : key;
        }
      }
      key = group_max_u64<NT, NW>(key, g, sm.red[3]);
      const int m = 0x7fffffff - (int)(key & 0xffffffffu);
      g.sync();
#pragma unroll
      for (int q = 0; q < RPT; ++q)
        if (t + q * NT == m) {
#pragma unroll
          for (int c = 0; c < KB; c += 2) {
            sm.vb[c] = Pr[q][c / 2].x;
            sm.vb[c + 1] = Pr[q][c / 2].y;
          }
        }
      g.sync();
      double zp = 0.0;
      float z[RPT];
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        z[q] = sm.vb[t + q * NT];
        zp += (double)z[q] * (double)z[q];
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
  g.sync();  // T visible to every thread
  if constexpr (PF) {
    pre.finish(stg, t);  // what the steps left (small k, early exit)
    *issued = pre.on;
  }

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
      if (m == 0) {
        sm.red[4][0] = e;
        if (out.lmin) out.lmin[set] = e;
      }
      if (m == k - 1) {
        sm.red[5][0] = e;
        if (out.lmax) out.lmax[set] = e;
      }
    }
    constexpr int W = NT < 32 ? NT : 32;
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) prod *= __shfl_xor_sync(g.mask, prod, o);
    if constexpr (NW > 1) {
      if ((threadIdx.x & 31) == 0) sm.red[0][g.wig] = prod;
    }
    g.sync();
    if (t == 0) {
      double det = prod;
      if constexpr (NW > 1) {
        det = sm.red[0][0];
        for (int w2 = 1; w2 < NW; ++w2) det *= sm.red[0][w2];
      }
      if (out.det) out.det[set] = det;
      if (out.delta) out.delta[set] = fmax(1.0 - sm.red[4][0], sm.red[5][0] - 1.0);
      if (out.err) out.err[set] = status;
    }
  }
  g.sync();
  return -1;
}

}  // namespace pl
