/*
 * pl_oracle.c -- CPU oracle for the subset-eigenvalue path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file.  Only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * reference arm of bench.py use it, and only as the checker / CPU baseline.
 *
 * What it restates (ParaLanczos v0.21, file:line within the reference project):
 *   - orc_ker2_lanczos   : the per-subset k-step Lanczos recurrence of
 *                          POS_SYM_SUBMATRIX_KER2, ParaLanczos.cu:1285-1374, with
 *                          the alpha/beta storage of ParaLanczos.cu:1371-1372 and
 *                          the pad of ParaLanczos.cu:1377-1378.  The start vector
 *                          is all-ones/sqrt(k) instead of the clock-seeded cuRAND
 *                          normal vector of ParaLanczos.cu:1196-1233.
 *   - orc_tqlrat         : EISPACK TQLRAT as used at ParaLanczos.cu:32-189
 *                          (rational QL, ascending eigenvalues, ierr = l+1 after
 *                          30 iterations).  Same operation order, so the result
 *                          is bit-identical to the reference source compiled for
 *                          the host (checked in tests against oracle/_ref).
 *   - orc_det_tridiag    : the continuant of ParaLanczos.cu:243-269, applied to
 *                          the post-TQLRAT arrays as at ParaLanczos.cu:1465.
 *   - orc_subset_solve   : the per-set driver of ParaLanczos.cu:1454-1478
 *                          (square beta, TQLRAT, det, eigenvalue write-out).
 *   - orc_gen_*          : the project's counter-based index-set generator
 *                          (the reference has none; its callers hand in
 *                          subIndex, ParaLanczos.cu:1843-1845).  Same bits as
 *                          the device generator in paralanczos_b200/csrc.
 *   - orc_dsg_b          : the subset Gram kernel DSG_B, ParaLanczos.cu:364-382
 *                          (subgrams[j + i*n] = sum_k Frame[S_i + k*N + off] *
 *                          Frame[S_j + k*N + off], FP64, k ascending), the spec
 *                          of the on-the-fly Gram form.
 *   - orc_upper_power    : UPPER_KER's norm estimate, ParaLanczos.cu:1484-1626
 *                          (10 power iterations, Upper = ||A v_9||), with the
 *                          all-ones start instead of the clock-seeded normal one.
 *   - orc_sturm_count /
 *     orc_bisect_*       : the FP64 Sturm-count bisection the GPU path uses in
 *                          place of TQLRAT (the reference's only Sturm code,
 *                          EIGVALS_BELOW at ParaLanczos.cu:519-552, skips
 *                          alpha[1] and is unused).  Restated here so the device
 *                          bisection can be checked on identical tridiagonals.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ParaLanczos0.h:14,32 redefines DBL_EPSILON (and so _EPSILON) as this
 * truncated decimal; TQLRAT's tolerance uses it (ParaLanczos.cu:76). */
#define ORC_TQL_EPS 2.220446e-16

/* ------------------------------------------------------------------------- */
/* EISPACK TQLRAT restated (ParaLanczos.cu:32-189).                            */
/* d[0..n-1]: diagonal in, eigenvalues (ascending) out.                        */
/* e2[0..n-1]: squared sub-diagonal in e2[1..n-1] (e2[0] ignored), destroyed. */
/* Returns 0, or l+1 when eigenvalue l needed more than 30 iterations.         */
/* ------------------------------------------------------------------------- */
int orc_tqlrat(int n, double *d, double *e2)
{
    if (n == 1) return 0;
    for (int i = 1; i < n; ++i) e2[i - 1] = e2[i];   /* shift sub-diagonal down */
    e2[n - 1] = 0.0;

    double f = 0.0, tnorm = 0.0, tol = 0.0, tol2 = 0.0;
    for (int l = 0; l < n; ++l) {
        int iter = 0;
        double h = fabs(d[l]) + sqrt(e2[l]);
        if (tnorm <= h) {                 /* running norm sets the tolerance */
            tnorm = h;
            tol = fabs(tnorm) * ORC_TQL_EPS;
            tol2 = tol * tol;
        }
        int m = l;                        /* first negligible e2 at or after l */
        while (m < n && !(e2[m] <= tol2)) ++m;

        if (m != l) {
            for (;;) {
                if (iter >= 30) return l + 1;
                ++iter;
                /* shift from the leading 2x2 */
                int l1 = l + 1;
                double s = sqrt(e2[l]);
                double g = d[l];
                double p = (d[l1] - g) / (2.0 * s);
                double r = sqrt(p * p + 1.0 * 1.0);
                double sgn = (p < 0) ? -1.0 : 1.0;
                d[l] = s / (p + fabs(r) * sgn);
                h = g - d[l];
                for (int i = l1; i < n; ++i) d[i] = d[i] - h;
                f = f + h;
                /* rational QL sweep from m-1 up to l */
                g = d[m];
                if (g == 0.0) g = tol;
                h = g;
                s = 0.0;
                for (int i = m - 1; i >= l; --i) {
                    p = g * h;
                    r = p + e2[i];
                    e2[i + 1] = s * r;
                    s = e2[i] / r;
                    d[i + 1] = h + s * (h + d[i]);
                    g = d[i] - e2[i] / g;
                    if (g == 0.0) g = tol;
                    h = g * p / r;
                }
                e2[l] = s * g;
                d[l] = h;
                if (h == 0.0) break;                       /* underflow guard */
                if (fabs(e2[l]) <= fabs(tol2 / h)) break;  /* converged */
                e2[l] = h * e2[l];
                if (e2[l] == 0.0) break;
            }
        }
        /* insert d[l]+f into the sorted prefix d[0..l] */
        double p = d[l] + f;
        int i = l;
        while (i > 0 && !(d[i - 1] <= p)) { d[i] = d[i - 1]; --i; }
        d[i] = p;
    }
    return 0;
}

/* Continuant f_n = a_n f_{n-1} - b_n^2 f_{n-2} (ParaLanczos.cu:243-269). */
double orc_det_tridiag(int n, const double *a, const double *b)
{
    double fm1 = 1.0, fm2 = 0.0, fn = 0.0;
    for (int i = 0; i < n; ++i) {
        fn = a[i] * fm1 - (b[i] * b[i]) * fm2;
        fm2 = fm1;
        fm1 = fn;
    }
    return fn;
}

typedef int (*orc_tqlrat_fn)(int, double *, double *);
typedef double (*orc_det_fn)(int, const double *, const double *);
static orc_tqlrat_fn g_tqlrat = orc_tqlrat;
static orc_det_fn g_det = orc_det_tridiag;

/* Swap in the reference's own compiled TQLRAT / DET_TRIDIAG (oracle/_ref). */
void orc_use_impl(orc_tqlrat_fn tq, orc_det_fn det)
{
    g_tqlrat = tq ? tq : orc_tqlrat;
    g_det = det ? det : orc_det_tridiag;
}

/* ------------------------------------------------------------------------- */
/* KER2 Lanczos recurrence restated in FP64 (ParaLanczos.cu:1285-1374).        */
/* As: k x k row-major.  alpha[0..k-1], beta[0..k+1] (beta[0]=0, beta[l+1] =   */
/* ||w_l||, beta[k+1]=0 pad).  No reorthogonalisation, as in the reference.    */
/* work: 4k doubles.                                                           */
/* ------------------------------------------------------------------------- */
void orc_ker2_lanczos(const double *As, int k, double *alpha, double *beta, double *work)
{
    double *v = work, *vprev = work + k, *y = work + 2 * k, *w = work + 3 * k;
    const double v0 = 1.0 / sqrt((double)k);
    for (int i = 0; i < k; ++i) { v[i] = v0; vprev[i] = 0.0; }
    beta[0] = 0.0;
    for (int l = 0; l < k; ++l) {
        for (int i = 0; i < k; ++i) {                 /* y = A v */
            double acc = 0.0;
            const double *row = As + (size_t)i * k;
            for (int c = 0; c < k; ++c) acc += row[c] * v[c];
            y[i] = acc;
        }
        double a = 0.0;
        for (int i = 0; i < k; ++i) a += v[i] * y[i];  /* alpha = v.Av */
        double bb = 0.0;
        for (int i = 0; i < k; ++i) {                   /* w = Av - (a v + beta_l vprev) */
            w[i] = y[i] - (a * v[i] + beta[l] * vprev[i]);
            bb += w[i] * w[i];
        }
        double b = sqrt(bb);
        for (int i = 0; i < k; ++i) { vprev[i] = v[i]; v[i] = w[i] / b; }
        beta[l + 1] = b;
        alpha[l] = a;
    }
    beta[k + 1] = 0.0;
}

/* Per-set driver (ParaLanczos.cu:1454-1478): gather A[S,S], Lanczos, square  */
/* beta, TQLRAT, det.  eig[0..k-1] ascending.  Returns TQLRAT's ierr.          */
/* A is float (a_is_double == 0) or double, row-major with leading dim lda.    */
/* Returns -1 when an index is out of [0, n).                                  */
int orc_subset_solve(const void *A, int a_is_double, int n, long long lda, const int *S, int k,
                     double *eig, double *det, double *work /* k*k + 8k + 4 */)
{
    double *As = work;
    double *alpha = As + (size_t)k * k;
    double *beta = alpha + k + 2;
    double *lw = beta + k + 2;
    for (int r = 0; r < k; ++r)
        if (S[r] < 0 || S[r] >= n) return -1;
    for (int r = 0; r < k; ++r)
        for (int c = 0; c < k; ++c) {
            size_t off = (size_t)S[r] * (size_t)lda + (size_t)S[c];
            As[(size_t)r * k + c] = a_is_double ? ((const double *)A)[off] : (double)((const float *)A)[off];
        }
    orc_ker2_lanczos(As, k, alpha, beta, lw);
    for (int i = 0; i < k + 2; ++i) beta[i] *= beta[i];
    int ierr = g_tqlrat(k, alpha, beta);
    double dt = g_det(k, alpha, beta);
    for (int i = 0; i < k; ++i) eig[i] = alpha[i];
    if (det) *det = dt;
    return ierr;
}

/* Batch over sets with OpenMP.  Uniform k when offsets == NULL (set s is      */
/* idx[s*k .. s*k+k-1]); CSR otherwise (set s is idx[offsets[s]..offsets[s+1]))*/
/* eig_all (nullable) gets k eigenvalues per set at the set's index offset.   */
void orc_batch(const void *A, int a_is_double, int n, long long lda, const int *idx,
               const long long *offsets, long long nsets, int k,
               double *lmin, double *lmax, double *delta, int *err,
               double *eig_all, double *det, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    int kmax = k;
    if (offsets) {
        kmax = 0;
        for (long long s = 0; s < nsets; ++s) {
            int ks = (int)(offsets[s + 1] - offsets[s]);
            if (ks > kmax) kmax = ks;
        }
    }
#pragma omp parallel
    {
        double *work = (double *)malloc(sizeof(double) * ((size_t)kmax * kmax + 8 * (size_t)kmax + 8));
        double *eig = (double *)malloc(sizeof(double) * ((size_t)kmax + 1));
#pragma omp for schedule(dynamic, 64)
        for (long long s = 0; s < nsets; ++s) {
            long long off = offsets ? offsets[s] : s * (long long)k;
            int ks = offsets ? (int)(offsets[s + 1] - offsets[s]) : k;
            double dt = 0.0;
            int ierr = orc_subset_solve(A, a_is_double, n, lda, idx + off, ks, eig, &dt, work);
            if (ierr < 0) {
                if (lmin) lmin[s] = NAN;
                if (lmax) lmax[s] = NAN;
                if (delta) delta[s] = NAN;
                if (err) err[s] = ierr;
                continue;
            }
            double lo = eig[0], hi = eig[ks - 1];
            if (lmin) lmin[s] = lo;
            if (lmax) lmax[s] = hi;
            if (delta) delta[s] = fmax(1.0 - lo, hi - 1.0);
            if (err) err[s] = ierr;
            if (det) det[s] = dt;
            if (eig_all) memcpy(eig_all + off, eig, sizeof(double) * (size_t)ks);
        }
        free(work);
        free(eig);
    }
}

/* ------------------------------------------------------------------------- */
/* Counter-based index-set generator (the project's own; no reference         */
/* counterpart).  Set s of a stream (seed) depends only on (seed, s).         */
/* ------------------------------------------------------------------------- */
uint64_t orc_splitmix64(uint64_t x)
{
    uint64_t z = x + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static uint64_t orc_set_key(uint64_t seed, uint64_t s)
{
    return orc_splitmix64(seed * 0x9E3779B97F4A7C15ULL + s);
}

static uint64_t orc_draw(uint64_t key, uint64_t i)
{
    return orc_splitmix64(key ^ (0x632BE59BD9B4E019ULL * (i + 1)));
}

static uint64_t orc_mulhi(uint64_t a, uint64_t b)
{
    return (uint64_t)(((unsigned __int128)a * (unsigned __int128)b) >> 64);
}

/* k distributions: 0 = fixed k; 1 = {8,16,24,32,48,64,96,128,192,256} with   */
/* P proportional to 1/k (integer weights 96,48,32,24,16,12,8,6,4,3 of 249); */
/* 2 = uniform in [kmin, kmax].                                              */
int orc_gen_k(uint64_t seed, uint64_t s, int kdist, int kmin, int kmax)
{
    if (kdist == 0) return kmin;
    uint64_t r = orc_draw(orc_set_key(seed, s), 0xFFFFFFFFULL);
    if (kdist == 1) {
        static const int kv[10] = {8, 16, 24, 32, 48, 64, 96, 128, 192, 256};
        static const int cum[10] = {96, 144, 176, 200, 216, 228, 236, 242, 246, 249};
        uint64_t u = orc_mulhi(r, 249);
        for (int i = 0; i < 10; ++i)
            if (u < (uint64_t)cum[i]) return kv[i];
        return 256;
    }
    return kmin + (int)orc_mulhi(r, (uint64_t)(kmax - kmin + 1));
}

/* Floyd's sampling of k distinct values in [0, n), in generation order. */
void orc_gen_set(uint64_t seed, uint64_t s, int n, int k, int *out)
{
    uint64_t key = orc_set_key(seed, s);
    for (int t = 0; t < k; ++t) {
        uint64_t j = (uint64_t)(n - k + t);
        uint64_t v = orc_mulhi(orc_draw(key, (uint64_t)t), j + 1);
        int dup = 0;
        for (int q = 0; q < t; ++q)
            if ((uint64_t)out[q] == v) { dup = 1; break; }
        out[t] = dup ? (int)j : (int)v;
    }
}

/* Fill a stream of sets.  offsets (nullable, nsets+1) receives CSR offsets;  */
/* idx receives the concatenated index sets.  Returns the total index count. */
long long orc_gen_stream(uint64_t seed, long long first, long long nsets, int n, int kdist, int kmin,
                         int kmax, long long *offsets, int *idx)
{
    long long off = 0;
    for (long long s = 0; s < nsets; ++s) {
        int k = orc_gen_k(seed, (uint64_t)(first + s), kdist, kmin, kmax);
        if (offsets) offsets[s] = off;
        if (idx) orc_gen_set(seed, (uint64_t)(first + s), n, k, idx + off);
        off += k;
    }
    if (offsets) offsets[nsets] = off;
    return off;
}

/* ------------------------------------------------------------------------- */
/* FP64 Sturm count and bisection (the GPU path's eigenvalue extraction).     */
/* alpha[0..k-1] diagonal; beta2[i] = beta_i^2 couples rows i-1 and i         */
/* (beta2[0] unused).  Counts eigenvalues of T strictly below x from sign     */
/* changes of the leading principal minors of T - xI (continuant form with    */
/* power-of-two rescaling; a zero minor is replaced by a tiny negative one).  */
/* ------------------------------------------------------------------------- */
int orc_sturm_count(const double *alpha, const double *beta2, int k, double x)
{
    double p0 = 1.0, p1 = alpha[0] - x;
    if (p1 == 0.0) p1 = -0x1p-900;
    int neg = p1 < 0.0;
    int cnt = neg;
    for (int i = 1; i < k; ++i) {
        double p2 = (alpha[i] - x) * p1 - beta2[i] * p0;
        if (p2 == 0.0) p2 = -0x1p-900 * fabs(p1);
        if (p2 == 0.0) p2 = -0x1p-1000;
        int n2 = p2 < 0.0;
        cnt += (n2 != neg);
        neg = n2;
        p0 = p1;
        p1 = p2;
        if ((i & 7) == 7) {
            double m = fmax(fabs(p0), fabs(p1));
            if (m > 0x1p200 || m < 0x1p-200) {
                int e;
                frexp(m, &e);
                p0 = ldexp(p0, -e);
                p1 = ldexp(p1, -e);
            }
        }
    }
    return cnt;
}

void orc_gershgorin(const double *alpha, const double *beta2, int k, double *lo, double *hi)
{
    double a = INFINITY, b = -INFINITY;
    for (int i = 0; i < k; ++i) {
        double r = (i > 0 ? sqrt(beta2[i]) : 0.0) + (i + 1 < k ? sqrt(beta2[i + 1]) : 0.0);
        a = fmin(a, alpha[i] - r);
        b = fmax(b, alpha[i] + r);
    }
    double pad = 2.0 * 2.220446049250313e-16 * fmax(fabs(a), fabs(b)) + 1e-300;
    *lo = a - pad;
    *hi = b + pad;
}

/* Eigenvalue number m (0-based, ascending) by plain bisection to width tol. */
double orc_bisect_one(const double *alpha, const double *beta2, int k, int m, double lo, double hi)
{
    double a = lo, b = hi;
    for (int it = 0; it < 200; ++it) {
        double tol = 0x1p-50 * fmax(fabs(a), fabs(b)) + 1e-300;
        if (b - a <= tol) break;
        double x = 0.5 * (a + b);
        if (x <= a || x >= b) break;
        if (orc_sturm_count(alpha, beta2, k, x) >= m + 1) b = x; else a = x;
    }
    return 0.5 * (a + b);
}

void orc_bisect_all(const double *alpha, const double *beta2, int k, double *eig)
{
    double lo, hi;
    orc_gershgorin(alpha, beta2, k, &lo, &hi);
    for (int m = 0; m < k; ++m) eig[m] = orc_bisect_one(alpha, beta2, k, m, lo, hi);
}

/* ------------------------------------------------------------------------- */
/* DSG_B restated (ParaLanczos.cu:364-382): the n x n Gram block of the frame */
/* columns `subset` (row-major M x N frame, column offset `off`), FP64 sums   */
/* over the frame rows in ascending order.                                    */
void orc_dsg_b(double *subgram, const double *frame, int M, int N, const int *subset, int n, int off)
{
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) {
            double val = 0.0;
            for (int k = 0; k < M; ++k)
                val += frame[subset[i] + (long long)k * N + off] * frame[subset[j] + (long long)k * N + off];
            subgram[j + i * n] = val;
        }
    }
}

/* ------------------------------------------------------------------------- */
/* UPPER_KER restated (ParaLanczos.cu:1484-1626): v = ones/sqrt(n); 10 times  */
/* w = A v, b = ||w||, v = w / b; returns the last b.  FP64, row-major A.     */
double orc_upper_power(const double *A, int n)
{
    double *v = (double *)malloc(sizeof(double) * n), *w = (double *)malloc(sizeof(double) * n);
    double b = 0.0;
    for (int i = 0; i < n; ++i) v[i] = 1.0 / sqrt((double)n);
    for (int it = 0; it < 10; ++it) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) {
            double acc = 0.0;
            for (int j = 0; j < n; ++j) acc += A[(long long)i * n + j] * v[j];
            w[i] = acc;
            s += acc * acc;
        }
        b = sqrt(s);
        for (int i = 0; i < n; ++i) v[i] = w[i] / b;
    }
    free(v);
    free(w);
    return b;
}
