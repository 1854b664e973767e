// pl_dropin.cu -- the ParaLanczos.h host entry points, B200-native.
//
// Same names, signatures (C++ linkage, so objects built against the
// reference's header link unchanged), argument meaning, output layout and
// validation messages as the reference (ParaLanczos.cu:1685-1863).  What is
// deliberately different:
//   * no cudaDeviceReset (ParaLanczos.cu:1700/1717, 1739/1760, 1783/1803,
//     1837/1858): the caller's CUDA context survives;
//   * the FP64 input is uploaded, converted to FP32 on the device and kept
//     there while later calls pass the same matrix (address, order and a
//     content hash; the reference re-uploads it every call,
//     ParaLanczos.cu:1845-1846), then solved by the batched engine (full
//     reorthogonalisation, all k eigenvalues by FP64 bisection); Det is the
//     product of the eigenvalues (the reference's KER path evaluates
//     DET_TRIDIAG over the full matrix order, ParaLanczos.cu:1138);
//   * calculate_subeigs3 solves every subIndexLen/subn set (the reference's
//     grid of subIndexLen/128 blocks skips a ragged tail, ParaLanczos.cu:1829);
//   * stdout lines of the reference only with PL_VERBOSE=1;
//   * PL_STRICT=0 lifts the reference's subn % 4 == 0 and subn <= 128 limits
//     (up to PL_KMAX).
// Each pl_* variant returns a status; the void C++ wrappers drop it.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#include "../../include/paralanczos.h"
#include "pl_internal.h"

namespace {

bool env_on(const char* name, bool dflt) {
  const char* v = getenv(name);
  if (!v || !*v) return dflt;
  return !(v[0] == '0' || v[0] == 'n' || v[0] == 'N' || v[0] == 'f' || v[0] == 'F');
}

// All-eigenvalue solve of nsets uniform-k sets of an FP64 host matrix: the
// matrix is uploaded and converted to FP32 on the device, and kept there
// while later calls pass the same matrix (pl_api.cu, api_solve_f64_host).
int solve_f64_host(const double* mat, int n, const int* subIndex, int nsets, int k, int form,
                   double* eig, double* det, int* err) {
  return pl::api_solve_f64_host(mat, n, subIndex, nsets, k, form, eig, det, err);
}

}  // namespace

extern "C" {

// calculate_subeigs3 (ParaLanczos.cu:1811-1863): subIndexLen/subn sets of size
// subn from subIndex; Eigenvalues[subIndexLen] (ascending per set), Det[sets].
int pl_calculate_subeigs3(double* mat, int subIndexLen, int matsize, double* Eigenvalues,
                          double* Det, int* subIndex, int subn) {
  const bool strict = env_on("PL_STRICT", true);
  if (strict) {
    if (subn % 4 != 0 || subn > 128) {
      fprintf(stderr, " 'int subn' must be divisible by 4, and less than or equal to 128! \n");
      return PL_EINVAL;
    }
    if (subIndexLen % 32 != 0) {
      fprintf(stderr, " 'subIndexLen' must be divisible by 32! \n");
      return PL_EINVAL;
    }
  }
  if (subn < 1 || subn > PL_KMAX || subn > matsize || subIndexLen < 0 || subIndexLen % subn != 0)
    return PL_EINVAL;
  if (!mat || !Eigenvalues || !Det || !subIndex || matsize <= 0) return PL_EINVAL;
  const bool verbose = env_on("PL_VERBOSE", false);
  if (verbose) printf("welcome to calculate subeigs2...\n");
  const int nsets = subIndexLen / subn;
  int rc = solve_f64_host(mat, matsize, subIndex, nsets, subn, PL_FORM_BATCHED, Eigenvalues, Det,
                          nullptr);
  if (rc) return rc;
  if (verbose)
    for (int i = 0; i < subIndexLen; i++) printf("%d eigenvalue: %g \n", i, Eigenvalues[i]);
  return PL_OK;
}

// calculate_subeigs (ParaLanczos.cu:1725-1765): one set of size subn;
// Eigenvalues[subn], *Det.  The reference warns (and carries on) when
// subn % 4 != 0 or n > 128.
int pl_calculate_subeigs(double* mat, int n, double* Eigenvalues, double* Det, int* subIndex,
                         int subn) {
  const bool strict = env_on("PL_STRICT", true);
  if (strict && (subn % 4 != 0 || n > 128))
    fprintf(stderr, " 'int n' must be divisible by 4, and less than or equal to 128! \n");
  if (subn < 1 || subn > PL_KMAX || subn > n || !mat || !Eigenvalues || !Det || !subIndex)
    return PL_EINVAL;
  const int form = subn <= 128 ? PL_FORM_PLAIN : PL_FORM_BATCHED;
  int rc = solve_f64_host(mat, n, subIndex, 1, subn, form, Eigenvalues, Det, nullptr);
  if (rc) return rc;
  if (env_on("PL_VERBOSE", false))
    for (int i = 0; i < subn; i++) printf("%d eigenvalue: %g \n", i, Eigenvalues[i]);
  return PL_OK;
}

// calculate_subeigs2 (ParaLanczos.cu:1768-1808): n indices, sets of size
// subn; Eigenvalues[n], Det[0] (the reference copies one determinant back).
int pl_calculate_subeigs2(double* mat, int n, int matsize, double* Eigenvalues, double* Det,
                          int* subIndex, int subn) {
  const bool strict = env_on("PL_STRICT", true);
  if (strict && (subn % 4 != 0 || n > 128))
    fprintf(stderr, " 'int n' must be divisible by 4, and less than or equal to 128! \n");
  const bool verbose = env_on("PL_VERBOSE", false);
  if (verbose) printf("welcome to calculate subeigs2...\n");
  if (subn < 1 || subn > PL_KMAX || subn > matsize || n < subn || !mat || !Eigenvalues || !Det ||
      !subIndex)
    return PL_EINVAL;
  const int nsets = n / subn;
  std::vector<double> det(nsets);
  std::vector<double> eig((size_t)nsets * subn);
  int rc = solve_f64_host(mat, matsize, subIndex, nsets, subn, PL_FORM_BATCHED, eig.data(),
                          det.data(), nullptr);
  if (rc) return rc;
  for (int i = 0; i < nsets * subn; ++i) Eigenvalues[i] = eig[i];
  Det[0] = det[0];
  if (verbose)
    for (int i = 0; i < n; i++) printf("%d eigenvalue: %g \n", i, Eigenvalues[i]);
  return PL_OK;
}

// calculate_eigs (ParaLanczos.cu:1685-1722): all eigenvalues of the n x n
// matrix; Eigenvalues[n], *Det.
int pl_calculate_eigs(double* mat, int n, double* Eigenvalues, double* Det) {
  const bool strict = env_on("PL_STRICT", true);
  if (strict && (n % 4 != 0 || n > 128))
    fprintf(stderr, " 'int n' must be divisible by 4, and less than or equal to 128! \n");
  if (n < 1 || n > PL_KMAX || !mat || !Eigenvalues || !Det) return PL_EINVAL;
  std::vector<int> S(n);
  for (int i = 0; i < n; ++i) S[i] = i;
  const int form = n <= 128 ? PL_FORM_PLAIN : PL_FORM_BATCHED;
  int rc = solve_f64_host(mat, n, S.data(), 1, n, form, Eigenvalues, Det, nullptr);
  if (rc) return rc;
  if (env_on("PL_VERBOSE", false))
    for (int i = 0; i < n; i++) printf("%d eigevalue: %g \n", i, Eigenvalues[i]);
  return PL_OK;
}

}  // extern "C"

// ---- C++ linkage drop-ins (ParaLanczos.h:39-47) ------------------------------
void print_tridiagonal(double* alpha, double* beta, int n) {
  // ParaLanczos.cu:1642-1682: MATLAB-style print of the tridiagonal whose
  // diagonal is alpha and whose off-diagonals are beta[1..n-1].
  printf(" [ ");
  for (int r = 0; r < n; r++) {
    for (int c = 0; c < n; c++) {
      double val = 0.0;
      if (r == c) val = alpha[c];
      else if (c == r - 1) val = beta[c + 1];
      else if (c == r + 1) val = beta[c];
      printf(" %g ", val);
      if (c != n - 1) printf(", ");
    }
    printf(r != n - 1 ? "; \n" : "] \n");
  }
}

void calculate_eigs(double* mat, int n, double* Eigenvalues, double* Det) {
  pl_calculate_eigs(mat, n, Eigenvalues, Det);
}

void calculate_subeigs(double* mat, int n, double* Eigenvalues, double* Det, int* subIndex,
                       int subn) {
  pl_calculate_subeigs(mat, n, Eigenvalues, Det, subIndex, subn);
}

void calculate_subeigs2(double* mat, int n, int matsize, double* Eigenvalues, double* Det,
                        int* subIndex, int subn) {
  pl_calculate_subeigs2(mat, n, matsize, Eigenvalues, Det, subIndex, subn);
}

void calculate_subeigs3(double* mat, int subIndexLen, int matsize, double* Eigenvalues,
                        double* Det, int* subIndex, int subn) {
  pl_calculate_subeigs3(mat, subIndexLen, matsize, Eigenvalues, Det, subIndex, subn);
}
