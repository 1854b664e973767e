/*
 * ParaLanczos.h -- source- and link-compatible drop-in for the host API of
 * ParaLanczos v0.21 (its ParaLanczos.h:39-47), implemented by
 * libparalanczos_b200.so on sm_100a.
 *
 * The declarations keep the reference's names, parameter lists and C++ linkage
 * so that objects compiled against the original header (example1.cu ..
 * example3.cu) link against this library unchanged; the mangled symbols are
 * _Z18calculate_subeigs3PdiiS_S_Pii and friends.  Behaviour per function is
 * documented in include/paralanczos.h (pl_calculate_*), which also gives the
 * status-returning C versions.  The reference's __global__ kernels
 * (its ParaLanczos.h:24-36) are declared below for CUDA translation units;
 * the library defines them with the same names and launch geometry (MATLAB's
 * CUDAKernel launches, see paralanczos_b200/csrc/pl_compat.cu).  A C caller
 * launches them through pl_launch_reference_kernel (include/paralanczos.h).
 */
#ifndef PARALANCZOS
#define PARALANCZOS

/* ParaLanczos.cu:1642-1682 -- prints the tridiagonal (alpha; beta[1..n-1]). */
void print_tridiagonal(double *alpha, double *beta, int n);

/* ParaLanczos.cu:1685-1722 -- all eigenvalues of an n x n matrix. */
void calculate_eigs(double *mat, int n, double *Eigenvalues, double *Det);

/* ParaLanczos.cu:1725-1765 -- eigenvalues of one subset of size subn. */
void calculate_subeigs(double *mat, int n, double *Eigenvalues, double *Det, int *subIndex, int subn);

/* ParaLanczos.cu:1768-1808 -- n indices in sets of subn (deprecated upstream). */
void calculate_subeigs2(double *mat, int n, int matsize, double *Eigenvalues, double *Det, int *subIndex, int subn);

/* ParaLanczos.cu:1811-1863 -- subIndexLen/subn sets of size subn. */
void calculate_subeigs3(double *mat, int subIndexLen, int matsize, double *Eigenvalues, double *Det, int *subIndex, int subn);

#ifdef __CUDACC__
/* ParaLanczos.h:24-36 -- kernels with the reference's names and parameters. */
__global__ void DSG_B(double *subgrams, double *Frame, int M, int N, int *subset, int n, int offset1);
__global__ void DSG_B1(double *subgrams, double *Frame, int M, int N, int *subset, int offset1);
__global__ void SG_B1(double *subgrams, double *Frame, int card);
__global__ void POS_SYM_MAT_KER(double *mat, int n, double *DetMat, double *Eigenvalues, int *Eigerror);
__global__ void POS_SYM_SUBMATRIX_KER(double *mat, int n, double *DetMat, double *Eigenvalues, int *Eigerror, int *subIndex, int subn);
__global__ void POS_SYM_SUBMATRIX_KER2(double *mat, int n, double *DetMat, double *Eigenvalues, int *Eigerror, int *subIndex, int subn);
__global__ void UPPER_KER(double *mat, int n, double *Upper);
#endif

#endif
