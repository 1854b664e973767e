// pl_cluster.cuh -- large-k per-set Lanczos on a thread-block cluster.
//
// For 128 < k <= 512 the per-set state (A_S and the projector P, 2 k^2 floats:
// 512 KB at k = 256, 2 MB at k = 512) does not fit one SM.  A cluster of CS
// CTAs (one per SM) holds one set: CTA c owns rows [c R, c R + R), R = KB/CS,
// with its rows of A_S in shared memory (lane-interleaved float4 layout) and
// its rows of P in registers.  Same recurrence as pl_engine.cuh (three-term
// step, w = P w~, P -= v v^T fused with the next matvec, FP32 vectors, FP64
// alpha/beta).  Per step the CTAs exchange, through distributed shared memory:
// their FP64 partials of alpha and ||w||^2 (every CTA sums the CS partials in
// rank order, so the scalars are bitwise identical cluster-wide and every
// branch is cluster-uniform), and their rows of w~ and w (written into every
// peer's broadcast buffers).  Two cluster barriers per step: one carries the
// rows of y = A v with the alpha partials (each CTA then forms all of
// w~ = y - alpha v_j - beta_j v_{j-1} locally), one carries the rows of w with
// the ||w||^2 partials.
//
// Thread mapping inside a CTA: NTC threads; a thread holds RPT of the CTA's
// R rows (rows ls, ls + R/RPT, ...), TPR = NTC * RPT / R threads share a row;
// thread g = t % TPR of a row owns the float4 column chunks g, g + TPR,
// g + 2 TPR, ... (CPT = KB / TPR columns of each of its rows), so the TPR
// threads of a row read adjacent 16-byte chunks of a broadcast vector:
// conflict-free shared-memory loads.  Row partial sums are combined with
// xor-shuffles over the TPR lanes (TPR divides 32).  With RPT = 2 a thread
// holds as much of P as with one row of twice the columns, but reads half of
// each broadcast vector per step.
#pragma once
#include <cooperative_groups.h>

#include "pl_engine.cuh"
#include "pl_sturm.cuh"

namespace pl {

namespace cg = cooperative_groups;

template <int KB, int CS, int NTC, int RPT = 1>
struct CfgC {
  static constexpr int R = KB / CS;       // rows per CTA
  static constexpr int RS = R / RPT;      // row slots: a thread holds rows ls, ls + RS, ...
  static constexpr int TPR = NTC / RS;    // threads per row
  static constexpr int CPT = KB / TPR;    // columns per thread (of each of its rows)
  static constexpr int NCH = CPT / 4;     // float4 chunks per thread and row
  static constexpr int NWC = NTC / 32;    // warps per CTA
  static_assert(KB % CS == 0 && R % RPT == 0 && NTC % RS == 0 && KB % TPR == 0, "bad shape");
  static_assert(32 % TPR == 0 && CPT % 4 == 0, "bad shape");
};

template <int KB, int CS, int NTC>
struct __align__(16) ClusterSmem {
  float4 A[(KB / CS) * KB / 4];  // own rows, [chunk][thread]
  float vb[3][KB];               // unnormalised Lanczos vectors, rotating: current, previous, next
  float yb[KB];                  // broadcast of y = A v
  float wb[KB];                  // w~, formed locally from yb
  int idx[KB];
  double2 ab[KB];                // T (rank 0 reads it for the bisection)
  double part[4][CS > NTC / 32 ? CS : NTC / 32];  // alpha, ||w||^2, misc, index check: rank
                                                // partials (warp partials for one CTA)
  double red[NTC / 32];          // warp partials inside the CTA
  unsigned long long key[CS];    // breakdown argmax exchange
};

// Barrier over the set's CTAs.  A one-CTA cluster needs only the CTA barrier
// (same ordering of its shared-memory writes, without the cluster-scope
// release/acquire).
template <int CS>
__device__ __forceinline__ void set_sync(cg::cluster_group& cl) {
  if constexpr (CS == 1)
    __syncthreads();
  else
    cl.sync();
}

// Sum over the CTA, then over the cluster (rank order).  Identical everywhere.
// A one-CTA set skips the CTA-level step: each warp's lane 0 stores its
// partial in part[slot][warp], one block barrier, and every thread adds the
// warps' partials in warp order.  (With several CTAs per set, the same scheme
// -- every warp storing into every peer -- measured slower than one CTA
// barrier plus one store per peer.)
template <int KB, int CS, int NTC>
__device__ __forceinline__ double cluster_sum(double x, ClusterSmem<KB, CS, NTC>& sm, int slot,
                                              cg::cluster_group& cl, int rank) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  const int w = threadIdx.x >> 5;
  if constexpr (CS == 1) {
    if ((threadIdx.x & 31) == 0) sm.part[slot][w] = x;
    __syncthreads();
    double s = sm.part[slot][0];
#pragma unroll
    for (int i = 1; i < NTC / 32; ++i) s += sm.part[slot][i];
    return s;
  } else {
    if ((threadIdx.x & 31) == 0) sm.red[w] = x;
    __syncthreads();
    if (threadIdx.x < CS) {
      double s = sm.red[0];
#pragma unroll
      for (int i = 1; i < NTC / 32; ++i) s += sm.red[i];
      ClusterSmem<KB, CS, NTC>* peer = cl.map_shared_rank(&sm, (unsigned)threadIdx.x);
      peer->part[slot][rank] = s;
    }
    set_sync<CS>(cl);
    double s = sm.part[slot][0];
#pragma unroll
    for (int r = 1; r < CS; ++r) s += sm.part[slot][r];
    return s;
  }
}

template <int KB, int CS, int NTC, int RPT = 1>
__device__ __forceinline__ void cluster_solve_set(const MatrixF32& M, const int* __restrict__ S,
                                                  int k, long long set, const SetOutputs& out,
                                                  ClusterSmem<KB, CS, NTC>& sm,
                                                  cg::cluster_group& cl, int rank) {
  using C = CfgC<KB, CS, NTC, RPT>;
  constexpr int R = C::R, RS = C::RS, TPR = C::TPR, CPT = C::CPT, NCH = C::NCH;
  const int t = threadIdx.x;
  const int ls = t / TPR;              // row slot: local rows ls + q * RS
  int r[RPT];                          // global rows
#pragma unroll
  for (int q = 0; q < RPT; ++q) r[q] = rank * R + ls + q * RS;
  const int g0 = t % TPR;              // owned chunks g0 + TPR * ch
  const bool lead = g0 == 0;
  const unsigned rmask = (TPR == 32) ? 0xffffffffu : (((1u << TPR) - 1u) << ((t & 31) / TPR * TPR));

  // ---- indices (every CTA keeps the full set), validation -------------------
  const SetMatrix SM = set_matrix(M, set);
  bool bad = false;
  for (int c = t; c < KB; c += NTC) {
    int v = 0;
    if (c < k) {
      v = SM.index(S, c);
      bad |= (v < 0) | (v >= SM.n);
    }
    sm.idx[c] = (c < k && v >= 0 && v < SM.n) ? v : 0;
  }
  const double badsum = cluster_sum<KB, CS, NTC>(__any_sync(0xffffffffu, bad) ? 1.0 : 0.0, sm, 3, cl, rank);
  if (badsum != 0.0) {
    if (rank == 0 && t == 0) write_failed(out, set, 0, 0, SET_BAD_INDEX);
    set_sync<CS>(cl);
    return;
  }

  // ---- gather own rows of A_S into shared memory; P = I ----------------------
  float4* __restrict__ my = sm.A + t;  // chunk (q, ch) at my[(q * NCH + ch) * NTC]
  float2 Pr[RPT][CPT / 2];
  double fro = 0.0;
  if constexpr (CS == 1) {
    // One CTA holds all of A_S, which is symmetric: load only its upper
    // triangle (k(k+1)/2 random elements, each its own L1 request) and store
    // each off-diagonal element twice.  Rows p and KB-1-p form a pair of KB+1
    // upper elements, shared by TPP threads.
    constexpr int NP = KB / 2, TPP = NTC / NP, PER = (KB + TPP) / TPP;
    static_assert(NP * TPP == NTC, "row pairs per CTA");
    float* __restrict__ Af = reinterpret_cast<float*>(sm.A);
    // float offset of element (row, col): chunk cc = col / 4 of row
    // q * RS + ls is held by thread ls * TPR + cc % TPR as its chunk (q, cc / TPR)
    auto at = [](int row, int col) {
      const int cc = col >> 2;
      return ((((row / RS) * NCH + cc / TPR) * NTC + (row % RS) * TPR + cc % TPR) << 2) + (col & 3);
    };
    const int p = t % NP, i0 = (t / NP) * PER;
    const int r0 = p, r1 = KB - 1 - p;
    const float* __restrict__ row0 = SM.A + (size_t)sm.idx[r0] * (size_t)SM.lda;
    const float* __restrict__ row1 = SM.A + (size_t)sm.idx[r1] * (size_t)SM.lda;
#pragma unroll 4
    for (int ii = 0; ii < PER; ++ii) {
      const int i = i0 + ii;
      if (i > KB) break;
      const bool first = i < KB - p;
      const int rr = first ? r0 : r1;
      const int c = first ? p + i : i - 1;  // c >= rr
      const float e = (rr < k && c < k) ? __ldg((first ? row0 : row1) + sm.idx[c]) : 0.f;
      const double e2 = (double)e * (double)e;
      fro += (c == rr) ? e2 : 2.0 * e2;
      Af[at(rr, c)] = e;
      if (c != rr) Af[at(c, rr)] = e;
    }
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const bool rv = r[q] < k;
#pragma unroll
      for (int ch = 0; ch < NCH; ++ch) {
        const int c = 4 * (g0 + TPR * ch);
        Pr[q][2 * ch] = make_float2((rv && c == r[q]) ? 1.f : 0.f, (rv && c + 1 == r[q]) ? 1.f : 0.f);
        Pr[q][2 * ch + 1] =
            make_float2((rv && c + 2 == r[q]) ? 1.f : 0.f, (rv && c + 3 == r[q]) ? 1.f : 0.f);
      }
    }
  } else {
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const bool rv = r[q] < k;
      const float* __restrict__ arow = SM.A + (size_t)sm.idx[r[q]] * (size_t)SM.lda;
#pragma unroll
      for (int ch = 0; ch < NCH; ++ch) {
        float e[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int c = 4 * (g0 + TPR * ch) + u;
          e[u] = (rv && c < k) ? __ldg(arow + sm.idx[c]) : 0.f;
          fro += (double)e[u] * (double)e[u];
        }
        my[(q * NCH + ch) * NTC] = make_float4(e[0], e[1], e[2], e[3]);
        const int c = 4 * (g0 + TPR * ch);
        Pr[q][2 * ch] = make_float2((rv && c == r[q]) ? 1.f : 0.f, (rv && c + 1 == r[q]) ? 1.f : 0.f);
        Pr[q][2 * ch + 1] =
            make_float2((rv && c + 2 == r[q]) ? 1.f : 0.f, (rv && c + 3 == r[q]) ? 1.f : 0.f);
      }
    }
  }
  const double fro2 = cluster_sum<KB, CS, NTC>(fro, sm, 2, cl, rank);
  const double tau2 = (32.0 * (double)kEps32) * (32.0 * (double)kEps32) * fro2;

  // vb[cur] holds the unnormalised v_j (v_j = sc * vb[cur]), vb[prv] v_{j-1}
  // (scaled by scp); w is published into vb[nxt].  Peers write vb[nxt] and yb
  // only after a cluster barrier that follows every read of the old contents.
  const float v0 = (float)(1.0 / sqrt((double)k));
  float v[RPT];
#pragma unroll
  for (int q = 0; q < RPT; ++q) v[q] = r[q] < k ? v0 : 0.f;
  for (int c = t; c < KB; c += NTC) {
    sm.vb[0][c] = c < k ? v0 : 0.f;
    sm.vb[1][c] = 0.f;
  }
  if (t == 0) sm.ab[0].y = 0.0;
  float sc = 1.f, scp = 0.f, bprev = 0.f;
  int status = 0;
  int cur = 0, prv = 1, nxt = 2;
  __syncthreads();

  for (int j = 0; j < k; ++j) {
    // P -= v v^T and y = A v over the owned row slices
    float2 ya[RPT], yb[RPT], nc[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const float cq = -v[q] * sc;
      nc[q] = make_float2(cq, cq);
      ya[q] = make_float2(0.f, 0.f);
      yb[q] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int ch = 0; ch < NCH; ++ch) {
      const float4 b4 = *reinterpret_cast<const float4*>(&sm.vb[cur][4 * (g0 + TPR * ch)]);
      const float2 b01 = make_float2(b4.x, b4.y), b23 = make_float2(b4.z, b4.w);
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const float4 a4 = my[(q * NCH + ch) * NTC];
        Pr[q][2 * ch] = __ffma2_rn(nc[q], b01, Pr[q][2 * ch]);
        Pr[q][2 * ch + 1] = __ffma2_rn(nc[q], b23, Pr[q][2 * ch + 1]);
        ya[q] = __ffma2_rn(make_float2(a4.x, a4.y), b01, ya[q]);
        yb[q] = __ffma2_rn(make_float2(a4.z, a4.w), b23, yb[q]);
      }
    }
    float y[RPT];
    double ap = 0.0;
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      y[q] = ((ya[q].x + ya[q].y) + (yb[q].x + yb[q].y)) * sc;
#pragma unroll
      for (int o = TPR / 2; o > 0; o >>= 1) y[q] += __shfl_xor_sync(rmask, y[q], o);
      ap = q == 0 ? (double)v[0] * (double)y[0] : fma((double)v[q], (double)y[q], ap);
    }
    // publish the owned rows of y with the alpha partial: one cluster barrier
    if (lead) {
#pragma unroll
      for (int p = 0; p < CS; ++p) {
        ClusterSmem<KB, CS, NTC>* peer = cl.map_shared_rank(&sm, (unsigned)p);
#pragma unroll
        for (int q = 0; q < RPT; ++q) peer->yb[r[q]] = y[q];
      }
    }
    const double alpha = cluster_sum<KB, CS, NTC>(lead ? ap : 0.0, sm, 0, cl, rank);
    const float af = (float)alpha;

    // w~ = y - alpha v_j - beta_j v_{j-1}, every element formed locally
    for (int c = t; c < KB; c += NTC)
      sm.wb[c] = fmaf(-af, sc * sm.vb[cur][c], fmaf(-bprev, scp * sm.vb[prv][c], sm.yb[c]));
    __syncthreads();

    // w = P w~ over the owned row slices
    float2 wa[RPT], wc[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      wa[q] = make_float2(0.f, 0.f);
      wc[q] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int ch = 0; ch < NCH; ++ch) {
      const float4 x4 = *reinterpret_cast<const float4*>(&sm.wb[4 * (g0 + TPR * ch)]);
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        wa[q] = __ffma2_rn(Pr[q][2 * ch], make_float2(x4.x, x4.y), wa[q]);
        wc[q] = __ffma2_rn(Pr[q][2 * ch + 1], make_float2(x4.z, x4.w), wc[q]);
      }
    }
    float w[RPT];
    double bp = 0.0;
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      w[q] = (wa[q].x + wa[q].y) + (wc[q].x + wc[q].y);
#pragma unroll
      for (int o = TPR / 2; o > 0; o >>= 1) w[q] += __shfl_xor_sync(rmask, w[q], o);
      bp = q == 0 ? (double)w[0] * (double)w[0] : fma((double)w[q], (double)w[q], bp);
    }
    if (lead) {
#pragma unroll
      for (int p = 0; p < CS; ++p) {
        ClusterSmem<KB, CS, NTC>* peer = cl.map_shared_rank(&sm, (unsigned)p);
#pragma unroll
        for (int q = 0; q < RPT; ++q) peer->vb[nxt][r[q]] = w[q];
      }
    }
    const double b2v = cluster_sum<KB, CS, NTC>(lead ? bp : 0.0, sm, 1, cl, rank);
    if (t == 0 && rank == 0) {
      sm.ab[j].x = alpha;
      if (j + 1 < k) sm.ab[j + 1].y = b2v;
    }
    if (!isfinite(alpha) || !isfinite(b2v)) {
      status |= SET_NONFINITE;
      break;
    }
    if (j + 1 == k) break;
    if (b2v > tau2) {
      const float bf = sqrtf((float)b2v);
      scp = sc;
      sc = 1.0f / bf;
      bprev = bf;
#pragma unroll
      for (int q = 0; q < RPT; ++q) v[q] = w[q] * sc;
    } else {
      // Breakdown: restart from the column of P with the largest diagonal
      // (cluster-wide argmax, ties to the smaller row), published into vb[nxt].
      status |= SET_BREAKDOWN;
      unsigned long long kk = 0ull;
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        if (r[q] < k && (r[q] >> 2) % TPR == g0) {  // this thread owns column r[q] of row r[q]
          float d = 0.f;
#pragma unroll
          for (int ch = 0; ch < NCH; ++ch) {
            const int c = 4 * (g0 + TPR * ch);
            if (c == r[q]) d = Pr[q][2 * ch].x;
            if (c + 1 == r[q]) d = Pr[q][2 * ch].y;
            if (c + 2 == r[q]) d = Pr[q][2 * ch + 1].x;
            if (c + 3 == r[q]) d = Pr[q][2 * ch + 1].y;
          }
          d = fmaxf(d, 0.f);
          const unsigned long long kq =
              ((unsigned long long)__float_as_uint(d) << 32) | (unsigned)(0x7fffffff - r[q]);
          kk = kq > kk ? kq : kk;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y2 = __shfl_xor_sync(0xffffffffu, kk, o);
        kk = y2 > kk ? y2 : kk;
      }
      if ((t & 31) == 0) sm.red[t >> 5] = __longlong_as_double((long long)kk);
      __syncthreads();
      if (t < CS) {
        unsigned long long m = 0;
        for (int i = 0; i < NTC / 32; ++i) {
          const unsigned long long y2 = (unsigned long long)__double_as_longlong(sm.red[i]);
          m = y2 > m ? y2 : m;
        }
        cl.map_shared_rank(&sm, (unsigned)t)->key[rank] = m;
      }
      set_sync<CS>(cl);
      unsigned long long best = 0;
#pragma unroll
      for (int q = 0; q < CS; ++q) best = sm.key[q] > best ? sm.key[q] : best;
      const int mrow = 0x7fffffff - (int)(best & 0xffffffffu);
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        if (r[q] == mrow) {
#pragma unroll
          for (int p = 0; p < CS; ++p) {
            float* dst = cl.map_shared_rank(&sm, (unsigned)p)->vb[nxt];
#pragma unroll
            for (int ch = 0; ch < NCH; ++ch) {
              const int c = 4 * (g0 + TPR * ch);
              dst[c] = Pr[q][2 * ch].x;
              dst[c + 1] = Pr[q][2 * ch].y;
              dst[c + 2] = Pr[q][2 * ch + 1].x;
              dst[c + 3] = Pr[q][2 * ch + 1].y;
            }
          }
        }
      }
      set_sync<CS>(cl);
      float z[RPT];
      double zp = 0.0;
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        z[q] = sm.vb[nxt][r[q]];
        zp = q == 0 ? (double)z[0] * (double)z[0] : fma((double)z[q], (double)z[q], zp);
      }
      const double zz = cluster_sum<KB, CS, NTC>(lead ? zp : 0.0, sm, 2, cl, rank);
      if (t == 0 && rank == 0) sm.ab[j + 1].y = 0x1p-600;  // decoupled block (see sturm_count)
      scp = sc;
      sc = 1.0f / sqrtf((float)zz);
      bprev = 0.f;
#pragma unroll
      for (int q = 0; q < RPT; ++q) v[q] = z[q] * sc;
    }
    const int old_prv = prv;
    prv = cur;
    cur = nxt;
    nxt = old_prv;
  }
  set_sync<CS>(cl);  // every rank done with the step loop before T is read

  // ---- extremes on rank 0: warp 0 lambda_min, warp 1 lambda_max, 33-way -----
  if (rank == 0) {
    if (status & SET_NONFINITE) {
      if (t == 0) write_failed(out, set, 0, 0, status);
    } else {
      double glo = 1e300, ghi = -1e300;
      if (t < 64) {
        for (int i = t & 31; i < k; i += 32) {
          const double rad = (i > 0 ? sqrt(sm.ab[i].y) : 0.0) + (i + 1 < k ? sqrt(sm.ab[i + 1].y) : 0.0);
          glo = fmin(glo, sm.ab[i].x - rad);
          ghi = fmax(ghi, sm.ab[i].x + rad);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          glo = fmin(glo, __shfl_xor_sync(0xffffffffu, glo, o));
          ghi = fmax(ghi, __shfl_xor_sync(0xffffffffu, ghi, o));
        }
        const double pad = 0x1p-51 * fmax(fabs(glo), fabs(ghi)) + 1e-300;
        const double e = multisect_warp(sm.ab, k, glo - pad, ghi + pad, t < 32 ? 1 : k);
        if ((t & 31) == 0) sm.part[2][t >> 5] = e;
      }
      __syncthreads();
      if (t == 0) {
        const double lmin = sm.part[2][0], lmax = sm.part[2][1];
        if (out.lmin) out.lmin[set] = lmin;
        if (out.lmax) out.lmax[set] = lmax;
        if (out.delta) out.delta[set] = fmax(1.0 - lmin, lmax - 1.0);
        if (out.err) out.err[set] = status;
      }
    }
  }
  set_sync<CS>(cl);  // rank 0's reads of T and part[] precede the next set's writes
}

}  // namespace pl
