// pl_cgs.cuh -- Lanczos with a stored basis and one classical Gram-Schmidt pass.
//
// Used by two forms:
//   * the plain one-set-per-block form (k <= 128): A_S and the basis V live in
//     shared memory; this is the straightforward B200 counterpart of
//     POS_SYM_SUBMATRIX_KER (ParaLanczos.cu:857-1154, one set per block) and the
//     comparator of the batched form;
//   * the large-k form (k > 128): A_S and V live in a per-CTA scratch slot in
//     global memory (L2-resident), streamed with coalesced loads.
// Each step: y = A v (symmetric A read by columns, coalesced), alpha = v.y,
// w~ = y - alpha v - beta_j v_{j-1} (ParaLanczos.cu:1329-1332), then one full
// CGS pass w = w~ - V (V^T w~), beta = ||w||, v = w / beta.  FP32 vectors,
// FP64 alpha/beta, FP64 Sturm bisection.
//
// Thread t owns rows t, t+NT, ... (RM rows at most).  Storage:
//   As[c*lda + i] = A_S[c][i] (= A_S[i][c]),  V[i*ldv + m] = element i of v_m.
#pragma once
#include "pl_engine.cuh"

namespace pl {

template <int KM, int NW>
struct __align__(16) CgsSmem {
  float vb[KM];
  float wb[KM];
  float hb[KM];
  int idx[KM];
  double2 ab[KM];  // T: ab[i] = {alpha_i, beta_i^2}
  double red[6][NW];
};

template <int NT, int RM, int KM, bool ALL>
__device__ __forceinline__ void cgs_solve_set(const MatrixF32& M, const int* __restrict__ S, int k,
                                              long long set, long long off, const SetOutputs& out,
                                              float* __restrict__ As, int lda,
                                              float* __restrict__ V, int ldv,
                                              CgsSmem<KM, (NT > 32 ? NT / 32 : 1)>& sm,
                                              const Grp<NT>& g) {
  constexpr int NW = NT > 32 ? NT / 32 : 1;
  const int t = g.t;

  const SetMatrix SM = set_matrix(M, set);
  bool bad = false;
  for (int c = t; c < k; c += NT) {
    const int v = SM.index(S, c);
    bad |= (v < 0) | (v >= SM.n);
    sm.idx[c] = (v >= 0 && v < SM.n) ? v : 0;
  }
  if (group_any<NT, NW>(bad, g, sm.red[3])) {
    if (t == 0) write_failed(out, set, off, ALL ? k : 0, SET_BAD_INDEX);
    g.sync();
    return;
  }
  g.sync();

  // gather A[S,S] (column c, row i) into As; Frobenius norm
  double fro = 0.0;
  for (int c = 0; c < k; ++c) {
    const float* __restrict__ arow = SM.A + (size_t)sm.idx[c] * (size_t)SM.lda;  // row S_c = column S_c
    for (int i = t; i < k; i += NT) {
      const float a = __ldg(arow + sm.idx[i]);
      As[(size_t)c * lda + i] = a;
      fro += (double)a * (double)a;
    }
  }
  const double fro2 = group_sum<NT, NW>(fro, g, sm.red[2]);
  const double tau = 32.0 * (double)kEps32 * sqrt(fro2);

  float v[RM], vp[RM];
  const float v0 = (float)(1.0 / sqrt((double)k));
#pragma unroll
  for (int q = 0; q < RM; ++q) {
    const int i = t + q * NT;
    v[q] = i < k ? v0 : 0.f;
    vp[q] = 0.f;
    if (i < k) {
      sm.vb[i] = v0;
      V[(size_t)i * ldv] = v0;
    }
  }
  float bprev = 0.f;
  int status = 0;
  g.sync();

  for (int j = 0; j < k; ++j) {
    // y = A v
    float y[RM];
#pragma unroll
    for (int q = 0; q < RM; ++q) y[q] = 0.f;
    for (int c = 0; c < k; ++c) {
      const float vc = sm.vb[c];
      const float* __restrict__ col = As + (size_t)c * lda;
#pragma unroll
      for (int q = 0; q < RM; ++q) {
        const int i = t + q * NT;
        if (i < k) y[q] = fmaf(col[i], vc, y[q]);
      }
    }
    double ap = 0.0;
#pragma unroll
    for (int q = 0; q < RM; ++q) ap += (double)v[q] * (double)y[q];
    const double alpha = group_sum<NT, NW>(ap, g, sm.red[0]);
    const float af = (float)alpha;

    float w[RM];
#pragma unroll
    for (int q = 0; q < RM; ++q) {
      const int i = t + q * NT;
      w[q] = fmaf(-af, v[q], fmaf(-bprev, vp[q], y[q]));
      if (i < k) sm.wb[i] = w[q];
    }
    g.sync();
    // h = V^T w~ over the j+1 stored vectors
#pragma unroll
    for (int q = 0; q < RM; ++q) {
      const int m = t + q * NT;
      if (m <= j) {
        float h = 0.f, h2 = 0.f;
        int i = 0;
        for (; i + 1 < k; i += 2) {
          h = fmaf(V[(size_t)i * ldv + m], sm.wb[i], h);
          h2 = fmaf(V[(size_t)(i + 1) * ldv + m], sm.wb[i + 1], h2);
        }
        if (i < k) h = fmaf(V[(size_t)i * ldv + m], sm.wb[i], h);
        sm.hb[m] = h + h2;
      }
    }
    g.sync();
    // w = w~ - V h
    double bp = 0.0;
#pragma unroll
    for (int q = 0; q < RM; ++q) {
      const int i = t + q * NT;
      if (i < k) {
        const float* __restrict__ vrow = V + (size_t)i * ldv;
        float acc = 0.f, acc2 = 0.f;
        int m = 0;
        for (; m + 1 <= j; m += 2) {
          acc = fmaf(vrow[m], sm.hb[m], acc);
          acc2 = fmaf(vrow[m + 1], sm.hb[m + 1], acc2);
        }
        if (m <= j) acc = fmaf(vrow[m], sm.hb[m], acc);
        w[q] -= (acc + acc2);
        bp += (double)w[q] * (double)w[q];
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
    for (int q = 0; q < RM; ++q) vp[q] = v[q];
    if (b2v > tau * tau) {
      const float bf = sqrtf((float)b2v);
      const float inv = 1.0f / bf;
      bprev = bf;
#pragma unroll
      for (int q = 0; q < RM; ++q) v[q] = w[q] * inv;
    } else {
      // Breakdown: restart from e_m projected off the basis, m the row of V
      // with the smallest norm (largest diagonal of I - V V^T).
      status |= SET_BREAKDOWN;
      unsigned long long key = 0ull;
#pragma unroll
      for (int q = 0; q < RM; ++q) {
        const int i = t + q * NT;
        if (i < k) {
          float rn = 0.f;
          for (int m = 0; m <= j; ++m) rn = fmaf(V[(size_t)i * ldv + m], V[(size_t)i * ldv + m], rn);
          const float d = fmaxf(1.f - rn, 0.f);
          const unsigned long long kk =
              ((unsigned long long)__float_as_uint(d) << 32) | (unsigned)(0x7fffffff - i);
          key = kk > key ? kk : key;
        }
      }
      key = group_max_u64<NT, NW>(key, g, sm.red[3]);
      const int mr = 0x7fffffff - (int)(key & 0xffffffffu);
      g.sync();
      for (int m = t; m <= j; m += NT) sm.hb[m] = V[(size_t)mr * ldv + m];
      g.sync();
      double zp = 0.0;
#pragma unroll
      for (int q = 0; q < RM; ++q) {
        const int i = t + q * NT;
        w[q] = 0.f;
        if (i < k) {
          float acc = 0.f;
          for (int m = 0; m <= j; ++m) acc = fmaf(V[(size_t)i * ldv + m], sm.hb[m], acc);
          w[q] = (i == mr ? 1.f : 0.f) - acc;
          zp += (double)w[q] * (double)w[q];
        }
      }
      const double zz = group_sum<NT, NW>(zp, g, sm.red[1]);
      if (t == 0) sm.ab[j + 1].y = 0x1p-600;  // decoupled block (see sturm_count)
      const float inv = 1.0f / sqrtf((float)zz);
      bprev = 0.f;
#pragma unroll
      for (int q = 0; q < RM; ++q) v[q] = w[q] * inv;
    }
    if constexpr (NW == 1) g.sync();  // everyone is done reading vb / V row data
#pragma unroll
    for (int q = 0; q < RM; ++q) {
      const int i = t + q * NT;
      if (i < k) {
        sm.vb[i] = v[q];
        V[(size_t)i * ldv + (j + 1)] = v[q];
      }
    }
    g.sync();
  }
  g.sync();

  if (status & SET_NONFINITE) {
    if (t == 0) write_failed(out, set, off, ALL ? k : 0, status);
    g.sync();
    return;
  }

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
  if constexpr (!ALL) {
    if constexpr (NW >= 2) {
      // warp 0 brackets lambda_min, warp 1 lambda_max, 33-way each
      if (g.wig < 2) {
        const double e = multisect_warp(sm.ab, k, glo, ghi, g.wig == 0 ? 1 : k);
        if ((threadIdx.x & 31) == 0) sm.red[4 + g.wig][0] = e;
      }
      g.sync();
      if (t == 0) {
        const double lmin = sm.red[4][0], lmax = sm.red[5][0];
        if (out.lmin) out.lmin[set] = lmin;
        if (out.lmax) out.lmax[set] = lmax;
        if (out.delta) out.delta[set] = fmax(1.0 - lmin, lmax - 1.0);
        if (out.err) out.err[set] = status;
      }
    } else {
      constexpr int GW = NT < 32 ? NT : 32;
      const int base = (NT < 32) ? ((threadIdx.x & 31) / NT) * NT : 0;
      const unsigned mask = (NT < 32) ? g.mask : 0xffffffffu;
      double lmin, lmax;
      multisect_extremes(sm.ab, k, glo, ghi, GW / 2, base, mask, lmin, lmax);
      if (t == 0) {
        if (out.lmin) out.lmin[set] = lmin;
        if (out.lmax) out.lmax[set] = lmax;
        if (out.delta) out.delta[set] = fmax(1.0 - lmin, lmax - 1.0);
        if (out.err) out.err[set] = status;
      }
    }
  } else {
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
}

}  // namespace pl
