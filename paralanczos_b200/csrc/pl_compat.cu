// pl_compat.cu -- the reference's __global__ entry points, under their own
// names, signatures and launch geometry.
//
// MATLAB's wrappers do not call the host API: they load the reference's PTX
// and launch its kernels themselves (Matlab/gpu_multi_subsvd2.m:59-65: grid
// L/128, block 32, subn = minor; gpu_multi_subsvd.m:54-60: grid L/minor,
// block minor/4; gpu_svd.m: one block of n/4 threads).  The kernels below keep
// the reference's C++ names and parameter lists (ParaLanczos.h:24-36), so the
// same launches work against this library's PTX (ParaLanczos.ptx, written by
// the build) or through pl_launch_reference_kernel from C:
//
//   POS_SYM_SUBMATRIX_KER2  128/subn sets per 32-thread block, subn/4 threads
//                           per set (ParaLanczos.cu:1157-1480)
//   POS_SYM_SUBMATRIX_KER   one set per block of subn/4 threads
//                           (ParaLanczos.cu:857-1154)
//   POS_SYM_MAT_KER         the whole n x n matrix in one block of n/4 threads
//                           (ParaLanczos.cu:556-853)
//   UPPER_KER               power-iteration estimate of ||A||_2
//                           (ParaLanczos.cu:1484-1626)
//   DSG_B, DSG_B1, SG_B1    Gram blocks of a frame (ParaLanczos.cu:364-438)
//
// Outputs keep the reference's layout: all subn eigenvalues of a set
// ascending at Eigenvalues[subn * set], DetMat[set], Eigerror[set].  MATLAB
// launches these kernels with no dynamic shared memory, so the subset kernels
// work in at most 48 KB of static shared memory: the set's submatrix is held
// as a packed FP32 upper triangle (33 KB at subn = 128), reduced to
// tridiagonal form by Householder reflections (FP32 storage, FP64 norms),
// and all eigenvalues come from the same FP64 Sturm bisection as the batched
// kernels.  (The batched kernels' register-resident Lanczos needs more state
// per set than a 32-thread block with 48 KB can hold.)  Eigerror carries the
// library's per-set status bits instead of TQLRAT's iteration count (0 =
// success in both).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "../../include/paralanczos.h"
#include "pl_common.cuh"
#include "pl_internal.h"
#include "pl_sturm.cuh"

namespace pl {
namespace compat {

constexpr int KMAXC = 128;                       // largest subn of the reference's kernels
constexpr int PACKED = KMAXC * (KMAXC + 1) / 2;  // 8256 floats

struct CompatSmem {
  float A[PACKED + 64];  // packed upper triangles of the block's sets
  float v[KMAXC];        // Householder vector, per set slices
  float q[KMAXC];        // p, then q = p - K v
  int ix[KMAXC];         // the sets' indices
  double2 ab[KMAXC];     // tridiagonal {d_i, e_{i-1}^2}
  double red[32];        // group partials (one slot per lane)
  double bc[32];         // group results (one slot per set)
};

// Row i of a packed upper triangle of order k starts at rs(i); A[i][j] (i <= j)
// is at rs(i) + j - i.
__device__ __forceinline__ int rs(int i, int k) { return i * k - (i * (i - 1)) / 2; }

// A group: G consecutive lanes of one warp working on one set.
struct Group {
  int t, G;
  unsigned mask;
  double* red;  // G slots
  double* bc;   // 1 slot
  __device__ __forceinline__ void sync() const { __syncwarp(mask); }
  // Deterministic sum over the group (lane order).
  __device__ __forceinline__ double sum(double x) const {
    red[t] = x;
    sync();
    if (t == 0) {
      double s = 0.0;
      for (int i = 0; i < G; ++i) s += red[i];
      *bc = s;
    }
    sync();
    return *bc;
  }
  __device__ __forceinline__ double max(double x) const {
    red[t] = x;
    sync();
    if (t == 0) {
      double s = red[0];
      for (int i = 1; i < G; ++i) s = fmax(s, red[i]);
      *bc = s;
    }
    sync();
    return *bc;
  }
};

__device__ __forceinline__ double nan64() { return __longlong_as_double(0x7ff8000000000000LL); }

// All k eigenvalues (ascending) and their product for the set S (identity:
// rows/columns 0..k-1) of the FP64 n x n matrix mat.
__device__ void compat_solve(const double* __restrict__ mat, int n, const int* __restrict__ S,
                             bool identity, int k, double* __restrict__ eig, double* __restrict__ det,
                             int* __restrict__ err, float* __restrict__ A, float* __restrict__ v,
                             float* __restrict__ q, int* __restrict__ ix, double2* __restrict__ ab,
                             const Group& g) {
  const int t = g.t, G = g.G;
  // ---- indices, validation, gather of the packed upper triangle ------------
  double bad = 0.0;
  for (int i = t; i < k; i += G) {
    const int s = identity ? i : S[i];
    ix[i] = s;
    if (s < 0 || s >= n) bad = 1.0;
  }
  if (g.max(bad) != 0.0) {
    for (int m = t; m < k; m += G) eig[m] = nan64();
    if (t == 0) {
      *det = nan64();
      *err = SET_BAD_INDEX;
    }
    return;
  }
  double nonfinite = 0.0;
  for (int i = t; i < k; i += G) {
    const double* __restrict__ row = mat + (size_t)ix[i] * (size_t)n;
    float* __restrict__ dst = A + rs(i, k) - i;
    for (int j = i; j < k; ++j) {
      const double x = row[ix[j]];
      if (!isfinite(x)) nonfinite = 1.0;
      dst[j] = (float)x;
    }
  }
  if (g.max(nonfinite) != 0.0) {
    for (int m = t; m < k; m += G) eig[m] = nan64();
    if (t == 0) {
      *det = nan64();
      *err = SET_NONFINITE;
    }
    return;
  }

  // ---- Householder reduction to tridiagonal form -----------------------------
  // Step j maps column j below the diagonal to alpha e_1 with
  // H = I - beta v v^T, then the trailing block B becomes H B H =
  // B - v q^T - q v^T with p = beta B v, q = p - (beta v.p / 2) v.
  for (int j = 0; j + 2 < k; ++j) {
    const float* __restrict__ rowj = A + rs(j, k) - j;  // rowj[i] = A[j][i], i >= j
    double s = 0.0;
    for (int i = j + 2 + t; i < k; i += G) s += (double)rowj[i] * (double)rowj[i];
    s = g.sum(s);
    const double x0 = rowj[j + 1];
    if (t == 0) ab[j].x = rowj[j];
    if (s == 0.0) {  // already tridiagonal in this column
      if (t == 0) ab[j + 1].y = x0 != 0.0 ? x0 * x0 : 0x1p-600;
      g.sync();
      continue;
    }
    const double nrm = sqrt(x0 * x0 + s);
    const double alpha = x0 >= 0.0 ? -nrm : nrm;
    const double v0 = x0 - alpha;
    const float beta = (float)(2.0 / (v0 * v0 + s));
    for (int i = j + 1 + t; i < k; i += G) v[i] = i == j + 1 ? (float)v0 : rowj[i];
    g.sync();
    double vp = 0.0;
    for (int i = j + 1 + t; i < k; i += G) {
      float acc = 0.f;
      for (int l = j + 1; l < i; ++l) acc = fmaf(A[rs(l, k) + i - l], v[l], acc);  // B(i,l) = A[l][i]
      const float* __restrict__ rowi = A + rs(i, k) - i;
      for (int l = i; l < k; ++l) acc = fmaf(rowi[l], v[l], acc);
      const float p = beta * acc;
      q[i] = p;
      vp += (double)v[i] * (double)p;
    }
    vp = g.sum(vp);
    const float K = (float)(0.5 * (double)beta * vp);
    for (int i = j + 1 + t; i < k; i += G) q[i] = fmaf(-K, v[i], q[i]);
    g.sync();
    for (int i = j + 1 + t; i < k; i += G) {
      const float vi = v[i], qi = q[i];
      float* __restrict__ rowi = A + rs(i, k) - i;
      for (int l = i; l < k; ++l) rowi[l] -= fmaf(vi, q[l], qi * v[l]);
    }
    if (t == 0) ab[j + 1].y = alpha * alpha;
    g.sync();
  }
  if (t == 0) {
    ab[0].y = 0.0;
    if (k >= 2) {
      const double e = A[rs(k - 2, k) + 1];
      ab[k - 2].x = A[rs(k - 2, k)];
      ab[k - 1].y = e != 0.0 ? e * e : 0x1p-600;
    }
    ab[k - 1].x = A[rs(k - 1, k)];
  }
  g.sync();

  // ---- all eigenvalues by FP64 Sturm bisection ---------------------------------
  double lo = 1e300, hi = -1e300;
  for (int i = t; i < k; i += G) {
    const double rad = (i > 0 ? sqrt(ab[i].y) : 0.0) + (i + 1 < k ? sqrt(ab[i + 1].y) : 0.0);
    lo = fmin(lo, ab[i].x - rad);
    hi = fmax(hi, ab[i].x + rad);
  }
  lo = -g.max(-lo);
  hi = g.max(hi);
  const double pad = 0x1p-51 * fmax(fabs(lo), fabs(hi)) + 1e-300;
  lo -= pad;
  hi += pad;
  int R = 0;
  {
    double w = hi - lo;
    const double tol = bisect_tol(lo, hi);
    while (w > tol && R < 200) {
      w *= 0.5;
      ++R;
    }
  }
  double prod = 1.0;
  for (int m = t; m < k; m += G) {
    const double e = bisect_index(ab, k, m, lo, hi, R);
    eig[m] = e;
    prod *= e;
  }
  // product over the group in lane order (deterministic)
  g.red[t] = prod;
  g.sync();
  if (t == 0) {
    double d = 1.0;
    for (int i = 0; i < G; ++i) d *= g.red[i];
    *det = d;
    *err = SET_OK;
  }
  g.sync();
}

__device__ __forceinline__ bool subn_ok(int subn) { return subn >= 4 && subn <= KMAXC && subn % 4 == 0; }

}  // namespace compat
}  // namespace pl

using namespace pl;
using namespace pl::compat;

// ---------------------------------------------------------------------------
// The reference's kernels (C++ linkage: the same mangled names).
// ---------------------------------------------------------------------------

// subn/4 threads per set, 128/subn sets per 32-thread block; set
// blockIdx.x * (32 / (subn / 4)) + subwarp (ParaLanczos.cu:1177-1190).
__global__ void POS_SYM_SUBMATRIX_KER2(double* mat, int n, double* DetMat, double* Eigenvalues,
                                       int* Eigerror, int* subIndex, int subn) {
  __shared__ CompatSmem sm;
  const int tx = threadIdx.x;
  if (!subn_ok(subn) || tx >= 32) return;
  const int G = subn / 4;
  const int nsw = 32 / G;
  const int sw = tx / G;
  if (sw >= nsw) return;  // lanes beyond the last whole subwarp
  const int t = tx - sw * G;
  const unsigned mask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (sw * G));
  const long long set = (long long)blockIdx.x * nsw + sw;
  const int k = subn;
  Group g{t, G, mask, sm.red + sw * G, sm.bc + sw};
  compat_solve(mat, n, subIndex + set * k, false, k, Eigenvalues + set * k, DetMat + set, Eigerror + set,
               sm.A + sw * (k * (k + 1) / 2), sm.v + sw * k, sm.q + sw * k, sm.ix + sw * k, sm.ab + sw * k, g);
}

// One set per block of subn/4 threads (ParaLanczos.cu:878-880).
__global__ void POS_SYM_SUBMATRIX_KER(double* mat, int n, double* DetMat, double* Eigenvalues, int* Eigerror,
                                      int* subIndex, int subn) {
  __shared__ CompatSmem sm;
  const int G = blockDim.x;
  if (!subn_ok(subn) || G != subn / 4 || G > 32) {
    if (threadIdx.x == 0) Eigerror[blockIdx.x] = SET_BAD_K;
    return;
  }
  const long long set = blockIdx.x;
  const unsigned mask = G == 32 ? 0xffffffffu : ((1u << G) - 1u);
  Group g{(int)threadIdx.x, G, mask, sm.red, sm.bc};
  compat_solve(mat, n, subIndex + set * subn, false, subn, Eigenvalues + set * subn, DetMat + set,
               Eigerror + set, sm.A, sm.v, sm.q, sm.ix, sm.ab, g);
}

// The whole n x n matrix, one block of n/4 threads (ParaLanczos.cu:556-853).
__global__ void POS_SYM_MAT_KER(double* mat, int n, double* DetMat, double* Eigenvalues, int* Eigerror) {
  __shared__ CompatSmem sm;
  const int G = blockDim.x;
  if (n < 1 || n > KMAXC || G > 32 || blockIdx.x != 0) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *Eigerror = SET_BAD_K;
    return;
  }
  const unsigned mask = G == 32 ? 0xffffffffu : ((1u << G) - 1u);
  Group g{(int)threadIdx.x, G, mask, sm.red, sm.bc};
  compat_solve(mat, n, nullptr, true, n, Eigenvalues, DetMat, Eigerror, sm.A, sm.v, sm.q, sm.ix, sm.ab, g);
}

// ||A||_2 estimate: 10 power iterations w = A v, Upper = ||w||, v = w / ||w||
// (ParaLanczos.cu:1484-1626).  The start vector is all-ones / sqrt(n) instead
// of the reference's clock-seeded normal vector.  Any block size; FP64.
__global__ void UPPER_KER(double* mat, int n, double* Upper) {
  __shared__ double vs[1024];
  __shared__ double ws[1024];
  __shared__ double red[1024];
  if (n < 1 || n > 1024 || blockIdx.x != 0) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *Upper = nan64();
    return;
  }
  const int T = blockDim.x;
  const int t = threadIdx.x;
  for (int i = t; i < n; i += T) vs[i] = 1.0 / sqrt((double)n);
  __syncthreads();
  double b = 0.0;
  for (int it = 0; it < 10; ++it) {
    double part = 0.0;
    for (int i = t; i < n; i += T) {
      const double* __restrict__ row = mat + (size_t)i * n;
      double acc = 0.0;
      for (int j = 0; j < n; ++j) acc = fma(row[j], vs[j], acc);
      ws[i] = acc;
      part += acc * acc;
    }
    red[t] = part;
    __syncthreads();
    if (t == 0) {
      double s = 0.0;
      for (int i = 0; i < T; ++i) s += red[i];
      red[0] = sqrt(s);
    }
    __syncthreads();
    b = red[0];
    for (int i = t; i < n; i += T) vs[i] = ws[i] / b;
    __syncthreads();
  }
  if (t == 0) *Upper = b;
}

// subgrams[j + i n] = sum_k Frame[subset[i] + k N + offset1] *
// Frame[subset[j] + k N + offset1]; thread (i, j) of an n x n block
// (ParaLanczos.cu:364-382).
__global__ void DSG_B(double* subgrams, double* Frame, int M, int N, int* subset, int n, int offset1) {
  const int i = threadIdx.x, j = threadIdx.y;
  if (i >= n || j >= n) return;
  const long long ci = subset[i] + (long long)offset1, cj = subset[j] + (long long)offset1;
  double val = 0.0;
  for (int r = 0; r < M; ++r) val += Frame[ci + (long long)r * N] * Frame[cj + (long long)r * N];
  subgrams[j + i * n] = val;
}

// Row i per thread of a blockDim.x-square Gram block (ParaLanczos.cu:388-406).
__global__ void DSG_B1(double* subgrams, double* Frame, int M, int N, int* subset, int offset1) {
  const int d = blockDim.x;
  const int i = threadIdx.x;
  const long long ci = subset[i] + (long long)offset1;
  for (int j = 0; j < d; ++j) {
    const long long cj = subset[j] + (long long)offset1;
    double val = 0.0;
    for (int r = 0; r < M; ++r) val += Frame[ci + (long long)r * N] * Frame[cj + (long long)r * N];
    subgrams[j + i * d] = val;
  }
}

// Gram of the first blockDim.x columns of a frame with row stride `card`,
// summed over its first blockDim.x rows (ParaLanczos.cu:410-438).
__global__ void SG_B1(double* subgrams, double* Frame, int card) {
  const int d = blockDim.x;
  const int i = threadIdx.x;
  for (int j = 0; j < d; ++j) {
    double val = 0.0;
    for (int r = 0; r < d; ++r) val += Frame[i + (long long)r * card] * Frame[j + (long long)r * card];
    subgrams[j + i * d] = val;
  }
}

extern "C" int pl_launch_reference_kernel(const char* name, unsigned grid_x, unsigned block_x,
                                          unsigned block_y, void** args, void* stream) {
  if (!name || !args || grid_x == 0 || block_x == 0 || block_y == 0) return PL_EINVAL;
  const void* fn = nullptr;
  if (!strcmp(name, "POS_SYM_SUBMATRIX_KER2")) fn = (const void*)POS_SYM_SUBMATRIX_KER2;
  else if (!strcmp(name, "POS_SYM_SUBMATRIX_KER")) fn = (const void*)POS_SYM_SUBMATRIX_KER;
  else if (!strcmp(name, "POS_SYM_MAT_KER")) fn = (const void*)POS_SYM_MAT_KER;
  else if (!strcmp(name, "UPPER_KER")) fn = (const void*)UPPER_KER;
  else if (!strcmp(name, "DSG_B")) fn = (const void*)DSG_B;
  else if (!strcmp(name, "DSG_B1")) fn = (const void*)DSG_B1;
  else if (!strcmp(name, "SG_B1")) fn = (const void*)SG_B1;
  else return PL_EINVAL;
  cudaError_t e = cudaLaunchKernel(fn, dim3(grid_x), dim3(block_x, block_y), args, 0, (cudaStream_t)stream);
  if (e != cudaSuccess) {
    api_note_cuda(e);
    return PL_ECUDA;
  }
  return PL_OK;
}
