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
 * status-returning C versions.  The reference's __global__ kernels are not
 * part of this header: their B200 replacements are reached through
 * pl_solve (include/paralanczos.h).
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

#endif
