// pl_common.cuh -- shared definitions for the sm_100a subset-eigenvalue kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pl {

// Per-set status bits written to err[] (the reference's Eigerror is TQLRAT's
// ierr, ParaLanczos.cu:1467; these extend it).
enum SetStatus : int {
  SET_OK = 0,
  SET_BREAKDOWN = 1,     // a Lanczos step had beta below the breakdown threshold;
                         // the recurrence was restarted (result still valid)
  SET_NONFINITE = 2,     // NaN/Inf met in the submatrix or the recurrence
  SET_BAD_INDEX = 4,     // an index of the set is outside [0, n)
  SET_BAD_K = 8,         // the set's k is outside the kernel's supported range
};

constexpr float kEps32 = 1.1920929e-7f;

// Where one launch reads its sets from.
struct SetSource {
  const int* idx;            // concatenated index sets (0-based rows/cols of A)
  const long long* offsets;  // CSR offsets (nsets+1) or nullptr for uniform k
  int k;                     // uniform k (offsets == nullptr)
  const int* perm;           // optional work-item -> set id map (binned queues)
  const int* perm_start;     // optional device-side offset of this queue in perm
  const int* count;          // optional device-side work-item count (binned queues)
  long long nitems;          // work items when count == nullptr
};

struct SetOutputs {
  double* lmin;   // lambda_min per set (nullable)
  double* lmax;   // lambda_max per set (nullable)
  double* delta;  // delta_k = max(1 - lambda_min, lambda_max - 1) (nullable)
  int* err;       // SetStatus bits (nullable)
  double* eig;    // all k eigenvalues ascending at the set's index offset (nullable)
  double* det;    // product of eigenvalues (nullable)
};

// One device-resident matrix of a table (serving: sets of one launch may
// name different matrices).
struct MatrixRef {
  const float* A;
  long long lda;
  int n;
};

struct MatrixF32 {
  const float* A;  // symmetric, row-major
  long long lda;
  int n;
  // > 0: A holds one already-formed k x k block per set (row stride lda) at
  // A + set * set_stride, indexed locally 0..k-1 (the on-the-fly Gram form);
  // n is then the block dimension.
  long long set_stride = 0;
  // non-null: set s reads matrix mats[mat_id[s]] instead of A / lda / n.
  const MatrixRef* mats = nullptr;
  const int* mat_id = nullptr;
};

// The matrix one set reads, resolved once at the start of its solve.
struct SetMatrix {
  const float* A;
  long long lda;
  int n;
  bool local;  // indices are block-local 0..k-1 (pre-formed block)
  // A set's indices are read once per solve: a streaming (evict-first) load,
  // so the index stream does not push the rows of A out of L2.
  __device__ __forceinline__ int index(const int* __restrict__ S, int c) const {
    return local ? c : __ldcs(S + c);
  }
};

__device__ __forceinline__ SetMatrix set_matrix(const MatrixF32& M, long long set) {
  if (M.mat_id) {
    const MatrixRef r = M.mats[__ldg(M.mat_id + set)];
    return SetMatrix{r.A, r.lda, r.n, false};
  }
  if (M.set_stride) return SetMatrix{M.A + set * M.set_stride, M.lda, M.n, true};
  return SetMatrix{M.A, M.lda, M.n, false};
}

__device__ __forceinline__ long long item_count(const SetSource& src) {
  return src.count ? (long long)(*src.count) : src.nitems;
}

__device__ __forceinline__ void set_span(const SetSource& src, long long item, int pbase,
                                         long long& set, long long& off, int& k) {
  set = src.perm ? (long long)src.perm[pbase + item] : item;
  if (src.offsets) {
    off = src.offsets[set];
    k = (int)(src.offsets[set + 1] - off);
  } else {
    off = set * (long long)src.k;
    k = src.k;
  }
}

}  // namespace pl
