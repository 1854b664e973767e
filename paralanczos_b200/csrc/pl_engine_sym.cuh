// pl_engine_sym.cuh -- one set per CTA with A_S and the projector P both kept
// as the upper triangle of 32 x 32 tiles.
//
// A_S and P are symmetric, so half of each is enough: for k = 256 the 36 upper
// tiles of A_S take 144 KB of shared memory and those of P 144 KB of registers,
// where the full matrices (512 KB together) need a 2-SM cluster and two
// cluster barriers per Lanczos step.  Same recurrence as pl_cluster.cuh and
// pl_engine.cuh (ParaLanczos.cu:1157-1480 with full reorthogonalisation in
// projector form): P -= v v^T fused with y = A v, w~ = y - alpha v_j -
// beta_j v_{j-1}, w = P w~, FP32 vectors, FP64 alpha and ||w||^2.
//
// Tile layout.  Tiles (I, J), I <= J, are numbered column by column over the
// upper triangle (t = J (J + 1) / 2 + I), so the tiles of a set with
// nb = ceil(k / 32) blocks are exactly t < nb (nb + 1) / 2.  Warp w holds tiles
// w, w + NW, ...  Lane l = 4 rg + cg holds 4 rows and 8 columns of a tile in
// 32 register slots: slot (a, s), a < 4, s < 8, is tile element
// (4 rg + (a ^ (cg & 2)), 8 cg + (s ^ (rg & 6))).  P lives in registers as 16
// slot pairs (a, 2p .. 2p + 1), two adjacent columns; A_S in shared memory as
// 8 float4 chunks (a, 4h .. 4h + 3) per lane, [tile][chunk][lane], so every
// chunk load is 512 contiguous bytes.  Diagonal tiles are held whole.
//
// A tile (I, J), I < J, contributes to two blocks of a product: its row sums
// (A_IJ x_J) to block I and its column sums (A_IJ^T x_I) to block J.  A lane's
// 4 row partials are reduced over the 4 lanes of its row group (3 shuffles;
// lane l ends with tile row l), its 8 column partials over the 8 lanes of its
// column group (7 shuffles; lane l ends with tile column 8 cg + rg).  The XOR
// in the slot order makes every level of these reduce-scatters but the last
// send its upper half of slots and keep its lower half, with no selects.
// Each tile writes its sums to ys[block][other block][32]; row i of the
// product is then the sum over the nb slots of its block, in block order
// (deterministic).  Per step: four CTA barriers (tile products, w~, tile
// products, w and ||w||^2).
#pragma once
#include "pl_engine.cuh"
#include "pl_sturm.cuh"

namespace pl {

template <int NB, int NW>
struct __align__(16) SymSmem {
  static constexpr int KB = 32 * NB, NT = NB * (NB + 1) / 2;
  float4 A[NT][8][32];  // upper tiles of A_S: [tile][chunk 2a + h][lane]
  float wb[3][KB];      // unnormalised Lanczos vectors, rotating: current, previous, next
  float wt[KB];         // w~
  float ys[NB][NB][32]; // tile sums: block, other block, row of the block
  double2 ab[KB];       // T: (alpha_j, beta_j^2)
  double pa[NW];        // alpha partials per warp
  double pb[NW];        // ||w||^2 partials per warp, and the Frobenius norm partials
  double pz[NW];        // norm partials of a breakdown restart vector
  unsigned long long key[NW];  // breakdown argmax per warp
  double ext[2];        // lambda_min, lambda_max
  int idx[KB];
};

// Sum over the warp; every lane gets the bitwise-same value (xor butterfly of
// commutative adds).
__device__ __forceinline__ double sym_warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// Sum of N partials in index order (every caller gets the bitwise-same value).
template <int N>
__device__ __forceinline__ double sym_sum(const double* p) {
  double s = p[0];
#pragma unroll
  for (int i = 1; i < N; ++i) s += p[i];
  return s;
}

// Slot (a, s) of lane (rg, cg): tile row and column.
__device__ __forceinline__ int sym_row(int rg, int cg, int a) { return 4 * rg + (a ^ (cg & 2)); }
__device__ __forceinline__ int sym_col(int rg, int cg, int s) { return 8 * cg + (s ^ (rg & 6)); }

// Row sums of the lanes' slots, reduced over the 4 lanes of a row group (lane
// bits 0-1): lane l ends with the sum of tile row l.  Level 1 pairs slot 0
// (1) with the partner's slot 2 (3): the same row.
__device__ __forceinline__ float sym_rows(const float (&rs)[4], int cg) {
  const float k0 = rs[0] + __shfl_xor_sync(0xffffffffu, rs[2], 2);
  const float k1 = rs[1] + __shfl_xor_sync(0xffffffffu, rs[3], 2);
  const bool o = cg & 1;
  const float keep = o ? k1 : k0, send = o ? k0 : k1;
  return keep + __shfl_xor_sync(0xffffffffu, send, 1);
}

// Column sums of the lanes' slots, reduced over the 8 lanes of a column group
// (lane bits 2-4): lane l = 4 rg + cg ends with tile column 8 cg + rg.
__device__ __forceinline__ float sym_cols(const float (&cs)[8], int rg) {
  float k4[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) k4[e] = cs[e] + __shfl_xor_sync(0xffffffffu, cs[4 + e], 16);
  float k2[2];
#pragma unroll
  for (int e = 0; e < 2; ++e) k2[e] = k4[e] + __shfl_xor_sync(0xffffffffu, k4[2 + e], 8);
  const bool o = rg & 1;
  const float keep = o ? k2[1] : k2[0], send = o ? k2[0] : k2[1];
  return keep + __shfl_xor_sync(0xffffffffu, send, 4);
}

// A block vector's values for the lane's slots: xI[a] = x[32 I + row(a)],
// xJ[p] = x[32 J + col(2p)], x[32 J + col(2p + 1)] (adjacent: float2 loads).
__device__ __forceinline__ void sym_load_vec(const float* __restrict__ x, int I, int J, int rg, int cg,
                                             float (&xI)[4], float2 (&xJ)[4]) {
  const float2 i0 = *reinterpret_cast<const float2*>(x + 32 * I + 4 * rg + (cg & 2));
  const float2 i1 = *reinterpret_cast<const float2*>(x + 32 * I + 4 * rg + (2 ^ (cg & 2)));
  xI[0] = i0.x;
  xI[1] = i0.y;
  xI[2] = i1.x;
  xI[3] = i1.y;
#pragma unroll
  for (int p = 0; p < 4; ++p) xJ[p] = *reinterpret_cast<const float2*>(x + 32 * J + 8 * cg + ((2 * p) ^ (rg & 6)));
}

// Tile t of the column-by-column numbering -> (I, J); t >= NT gives I = J = NB.
template <int NB>
__device__ __forceinline__ void sym_tile(int t, int& I, int& J) {
  I = NB;
  J = NB;
#pragma unroll
  for (int j = 0; j < NB; ++j) {
    const int first = j * (j + 1) / 2;
    if (t >= first && t < first + j + 1) {
      I = t - first;
      J = j;
    }
  }
}

// One tile's row and column partials of a product with x: m[a * 4 + p] holds
// slots (a, 2p .. 2p + 1); rs[a] = the slot row's partial over the lane's 8
// columns, cs[s] = the slot column's partial over its 4 rows (off-diagonal
// tiles only).
__device__ __forceinline__ void sym_tile_product(const float2 (&m)[16], const float (&xI)[4],
                                                 const float2 (&xJ)[4], bool diag, float (&rs)[4],
                                                 float (&cs)[8]) {
  float2 r2[4], c2[4];
#pragma unroll
  for (int a = 0; a < 4; ++a) r2[a] = make_float2(0.f, 0.f);
#pragma unroll
  for (int p = 0; p < 4; ++p) c2[p] = make_float2(0.f, 0.f);
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const float2 xa = make_float2(xI[a], xI[a]);
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      r2[a] = __ffma2_rn(m[a * 4 + p], xJ[p], r2[a]);
      if (!diag) c2[p] = __ffma2_rn(m[a * 4 + p], xa, c2[p]);
    }
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) rs[a] = r2[a].x + r2[a].y;
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    cs[2 * p] = c2[p].x;
    cs[2 * p + 1] = c2[p].y;
  }
}

// Tile sums of P x (x = sm.wt) for the warp's active tiles, into sm.ys.
template <int NB, int NW, int TPW>
__device__ __forceinline__ void sym_p_product(const float2 (&P)[TPW][16], SymSmem<NB, NW>& sm,
                                              const int (&TI)[TPW], const int (&TJ)[TPW], int nb, int lane) {
  const int rg = lane >> 2, cg = lane & 3;
#pragma unroll
  for (int u = 0; u < TPW; ++u) {
    if (TJ[u] >= nb) continue;  // warp-uniform
    const int I = TI[u], J = TJ[u];
    const bool diag = I == J;
    float xI[4];
    float2 xJ[4];
    sym_load_vec(sm.wt, I, J, rg, cg, xI, xJ);
    float rs[4], cs[8];
    sym_tile_product(P[u], xI, xJ, diag, rs, cs);
    sm.ys[I][J][lane] = sym_rows(rs, cg);
    if (!diag) sm.ys[J][I][8 * cg + rg] = sym_cols(cs, rg);
  }
}

template <int NB, int NW, int TPW>
__device__ __forceinline__ void sym_solve_set(const MatrixF32& M, const int* __restrict__ S, int k,
                                              long long set, const SetOutputs& out, SymSmem<NB, NW>& sm,
                                              const int (&TI)[TPW], const int (&TJ)[TPW],
                                              const int (&TT)[TPW]) {
  constexpr int KB = 32 * NB, NTH = NW * 32;
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const int rg = lane >> 2, cg = lane & 3;
  const int nb = (k + 31) >> 5;

  // ---- indices, validation -----------------------------------------------------
  const SetMatrix SM = set_matrix(M, set);
  int bad = 0;
  for (int c = t; c < KB; c += NTH) {
    int v = 0;
    if (c < k) {
      v = SM.index(S, c);
      bad |= (v < 0) | (v >= SM.n);
    }
    sm.idx[c] = (c < k && v >= 0 && v < SM.n) ? v : 0;
  }
  if (__syncthreads_or(bad)) {
    if (t == 0) write_failed(out, set, 0, 0, SET_BAD_INDEX);
    return;
  }

  // ---- gather the upper tiles of A_S; P = I -----------------------------------
  float2 P[TPW][16];
  double fro = 0.0;
#pragma unroll
  for (int u = 0; u < TPW; ++u) {
    const bool act = TJ[u] < nb;
    const bool diag = TI[u] == TJ[u];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int rl = sym_row(rg, cg, a), r = 32 * TI[u] + rl;
      const bool rv = act && r < k;
      const float* __restrict__ row = SM.A + (size_t)sm.idx[rv ? r : 0] * (size_t)SM.lda;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        float e[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int c = 32 * TJ[u] + sym_col(rg, cg, 4 * h + q);
          e[q] = (rv && c < k) ? __ldg(row + sm.idx[c]) : 0.f;
          const double e2 = (double)e[q] * (double)e[q];
          fro += diag ? e2 : 2.0 * e2;
        }
        if (act) sm.A[TT[u]][2 * a + h][lane] = make_float4(e[0], e[1], e[2], e[3]);
#pragma unroll
        for (int p = 0; p < 2; ++p) {
          const int cl = sym_col(rg, cg, 4 * h + 2 * p);  // cl + 1 is slot 4h + 2p + 1's column
          P[u][a * 4 + 2 * h + p] = make_float2((rv && diag && cl == rl) ? 1.f : 0.f,
                                                (rv && diag && cl + 1 == rl) ? 1.f : 0.f);
        }
      }
    }
  }
  fro = sym_warp_sum(fro);
  if (lane == 0) sm.pb[w] = fro;
  const float v0 = (float)(1.0 / sqrt((double)k));
  for (int c = t; c < KB; c += NTH) {
    sm.wb[0][c] = c < k ? v0 : 0.f;
    sm.wb[1][c] = 0.f;
  }
  if (t == 0) sm.ab[0].y = 0.0;
  __syncthreads();
  const double fro2 = sym_sum<NW>(sm.pb);
  const double tau2 = (32.0 * (double)kEps32) * (32.0 * (double)kEps32) * fro2;

  float sc = 1.f, scp = 0.f, bprev = 0.f;
  int status = 0;
  int cur = 0, prv = 1, nxt = 2;
  // Every warp has read pb[] (the norm partials) before phase D rewrites it:
  // phase D of step 0 follows three more barriers.

  for (int j = 0; j < k; ++j) {
    // ---- A: P -= v v^T, tile sums of y = A v, alpha partials -----------------
    double ap = 0.0;
    const float sc2 = sc * sc;
#pragma unroll
    for (int u = 0; u < TPW; ++u) {
      if (TJ[u] >= nb) continue;  // warp-uniform
      const int I = TI[u], J = TJ[u];
      const bool diag = I == J;
      // unnormalised w_j: v_j = sc w_j, so P -= sc^2 w w^T and the sums are scaled by sc
      float wI[4];
      float2 wJ[4];
      sym_load_vec(sm.wb[cur], I, J, rg, cg, wI, wJ);
      float2 r2[4], c2[4];
#pragma unroll
      for (int p = 0; p < 4; ++p) c2[p] = make_float2(0.f, 0.f);
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const float na = -sc2 * wI[a];
        const float2 nv = make_float2(na, na), xa = make_float2(wI[a], wI[a]);
        r2[a] = make_float2(0.f, 0.f);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const float4 a4 = sm.A[TT[u]][2 * a + h][lane];
          const float2 m0 = make_float2(a4.x, a4.y), m1 = make_float2(a4.z, a4.w);
          P[u][a * 4 + 2 * h] = __ffma2_rn(nv, wJ[2 * h], P[u][a * 4 + 2 * h]);
          P[u][a * 4 + 2 * h + 1] = __ffma2_rn(nv, wJ[2 * h + 1], P[u][a * 4 + 2 * h + 1]);
          r2[a] = __ffma2_rn(m0, wJ[2 * h], r2[a]);
          r2[a] = __ffma2_rn(m1, wJ[2 * h + 1], r2[a]);
          if (!diag) {
            c2[2 * h] = __ffma2_rn(m0, xa, c2[2 * h]);
            c2[2 * h + 1] = __ffma2_rn(m1, xa, c2[2 * h + 1]);
          }
        }
      }
      float rs[4], cs[8];
#pragma unroll
      for (int a = 0; a < 4; ++a) rs[a] = r2[a].x + r2[a].y;
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        cs[2 * p] = c2[p].x;
        cs[2 * p + 1] = c2[p].y;
      }
      // w_I^T (A w)_I over the lane's slots (FP32, 4 terms), accumulated in FP64
      const float af = fmaf(wI[3], rs[3], fmaf(wI[2], rs[2], fmaf(wI[1], rs[1], wI[0] * rs[0])));
      ap += diag ? (double)af : 2.0 * (double)af;
      sm.ys[I][J][lane] = sc * sym_rows(rs, cg);
      if (!diag) sm.ys[J][I][8 * cg + rg] = sc * sym_cols(cs, rg);
    }
    ap = sym_warp_sum(ap) * ((double)sc * (double)sc);
    if (lane == 0) sm.pa[w] = ap;
    __syncthreads();

    // ---- B: alpha, w~ = y - alpha v_j - beta_j v_{j-1} (the row warps) ---------
    if (t < KB) {
      const double alpha = sym_sum<NW>(sm.pa);
      const float af = (float)alpha;
      const int I = t >> 5;
      float y = 0.f;
      if (I < nb)
        for (int J = 0; J < nb; ++J) y += sm.ys[I][J][lane];
      sm.wt[t] = fmaf(-af, sc * sm.wb[cur][t], fmaf(-bprev, scp * sm.wb[prv][t], y));
      if (t == 0) sm.ab[j].x = alpha;
    }
    if (j + 1 == k) break;  // a non-finite alpha shows in ||w||^2 (or, at the end, in T)
    __syncthreads();

    // ---- C: tile sums of w = P w~ -----------------------------------------------
    sym_p_product<NB, NW, TPW>(P, sm, TI, TJ, nb, lane);
    __syncthreads();

    // ---- D: w, ||w||^2 ------------------------------------------------------------
    if (t < KB) {
      const int I = t >> 5;
      float wv = 0.f;
      if (I < nb)
        for (int J = 0; J < nb; ++J) wv += sm.ys[I][J][lane];
      sm.wb[nxt][t] = wv;
      const double bp = sym_warp_sum((double)wv * (double)wv);
      if (lane == 0) sm.pb[w] = bp;
    }
    __syncthreads();
    const double b2v = sym_sum<NB>(sm.pb);
    if (t == 0) sm.ab[j + 1].y = b2v;
    if (!isfinite(b2v)) {
      status |= SET_NONFINITE;
      break;
    }
    if (b2v > tau2) {
      const float bf = sqrtf((float)b2v);
      scp = sc;
      sc = 1.0f / bf;
      bprev = bf;
    } else {
      // Breakdown: restart from the column of P with the largest diagonal
      // (ties to the smaller row), written into wb[nxt].
      status |= SET_BREAKDOWN;
      unsigned long long kk = 0ull;
#pragma unroll
      for (int u = 0; u < TPW; ++u) {
        if (TJ[u] >= nb || TI[u] != TJ[u]) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int rl = sym_row(rg, cg, a), cl = sym_col(rg, cg, 2 * p + e), r = 32 * TI[u] + rl;
              if (rl == cl && r < k) {
                const float d = fmaxf(e ? P[u][a * 4 + p].y : P[u][a * 4 + p].x, 0.f);
                const unsigned long long kq =
                    ((unsigned long long)__float_as_uint(d) << 32) | (unsigned)(0x7fffffff - r);
                kk = kq > kk ? kq : kk;
              }
            }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y2 = __shfl_xor_sync(0xffffffffu, kk, o);
        kk = y2 > kk ? y2 : kk;
      }
      if (lane == 0) sm.key[w] = kk;
      __syncthreads();
      unsigned long long best = 0ull;
#pragma unroll
      for (int q = 0; q < NW; ++q) best = sm.key[q] > best ? sm.key[q] : best;
      const int mrow = 0x7fffffff - (int)(best & 0xffffffffu);
      // column mrow of P = P e_mrow, by the tile product (exact: one 1, zeros)
      if (t < KB) sm.wt[t] = t == mrow ? 1.f : 0.f;
      __syncthreads();
      sym_p_product<NB, NW, TPW>(P, sm, TI, TJ, nb, lane);
      __syncthreads();
      if (t < KB) {
        const int I = t >> 5;
        float z = 0.f;
        if (I < nb)
          for (int J = 0; J < nb; ++J) z += sm.ys[I][J][lane];
        sm.wb[nxt][t] = z;
        const double zp = sym_warp_sum((double)z * (double)z);
        if (lane == 0) sm.pz[w] = zp;
      }
      __syncthreads();
      const double zz = sym_sum<NB>(sm.pz);
      if (t == 0) sm.ab[j + 1].y = 0x1p-600;  // decoupled block (see sturm_count)
      scp = sc;
      sc = 1.0f / sqrtf((float)zz);
      bprev = 0.f;
    }
    const int old_prv = prv;
    prv = cur;
    cur = nxt;
    nxt = old_prv;
  }
  __syncthreads();  // T complete
  if (!isfinite(sm.ab[k - 1].x)) status |= SET_NONFINITE;  // the last alpha

  // ---- extremes: warp 0 lambda_min, warp 1 lambda_max, 33-way multisection ------
  if (status & SET_NONFINITE) {
    if (t == 0) write_failed(out, set, 0, 0, status);
  } else {
    if (t < 64) {
      double glo = 1e300, ghi = -1e300;
      for (int i = lane; i < k; i += 32) {
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
      if (lane == 0) sm.ext[w] = e;
    }
    __syncthreads();
    if (t == 0) {
      const double lmin = sm.ext[0], lmax = sm.ext[1];
      if (out.lmin) out.lmin[set] = lmin;
      if (out.lmax) out.lmax[set] = lmax;
      if (out.delta) out.delta[set] = fmax(1.0 - lmin, lmax - 1.0);
      if (out.err) out.err[set] = status;
    }
  }
  __syncthreads();  // the next set's writes follow every read of this one's state
}

}  // namespace pl
