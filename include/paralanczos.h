/*
 * paralanczos.h -- C ABI of the B200 (sm_100a) subset-eigenvalue library
 * libparalanczos_b200.so.
 *
 * Computes, for many index sets S of one symmetric matrix A, the eigenvalues
 * of the principal submatrix A[S,S] by a k-step Lanczos (start vector
 * all-ones/sqrt(k), FP32 vectors, FP64 alpha/beta, full reorthogonalisation)
 * and FP64 Sturm bisection of the tridiagonal, plus the restricted-isometry
 * constant delta_k = max(1 - lambda_min, lambda_max - 1).
 *
 * Every function returns a PL_* status (0 = success).  Device-pointer
 * functions are asynchronous on `stream` (a cudaStream_t passed as void*,
 * NULL = legacy default stream); host-pointer functions are synchronous.
 * Plain pointers and sizes only: no C++ or framework types cross this ABI.
 *
 * Reference interfaces replaced (ParaLanczos v0.21, file:line in that project):
 *   pl_solve / pl_solve_host       POS_SYM_SUBMATRIX_KER2 launched by
 *                                  calculate_subeigs3 (ParaLanczos.cu:1157-1480,
 *                                  1811-1863) and POS_SYM_SUBMATRIX_KER
 *                                  (ParaLanczos.cu:857-1154) as MATLAB launches
 *                                  them (Matlab/gpu_multi_subsvd*.m)
 *   pl_calculate_subeigs3          calculate_subeigs3, ParaLanczos.h:47,
 *                                  ParaLanczos.cu:1811-1863
 *   pl_calculate_subeigs           calculate_subeigs, ParaLanczos.h:43,
 *                                  ParaLanczos.cu:1725-1765
 *   pl_calculate_subeigs2          calculate_subeigs2, ParaLanczos.h:45,
 *                                  ParaLanczos.cu:1768-1808
 *   pl_calculate_eigs              calculate_eigs, ParaLanczos.h:41,
 *                                  ParaLanczos.cu:1685-1722
 *   pl_gen_sets / pl_gen_stream_host  no counterpart: the reference's callers
 *                                  build subIndex themselves (example2.cu:42-48)
 * The C++ (name-mangled) drop-in symbols of ParaLanczos.h are declared in
 * include/ParaLanczos.h and exported by the same library.
 */
#ifndef PARALANCZOS_B200_H
#define PARALANCZOS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define PL_OK 0
#define PL_EINVAL 1     /* bad argument (pointer, size, k)                    */
#define PL_ECUDA 2      /* a CUDA runtime call failed (pl_last_cuda_error)     */
#define PL_ENOMEM 3     /* device or pinned allocation failed                 */
#define PL_ENOTSUP 4    /* configuration not supported (e.g. k > PL_KMAX)     */
#define PL_ETIMEDOUT 5  /* a bounded device-side wait gave up                  */
#define PL_EBUSY 6      /* resource in use (serving queue full)               */

/* ---- per-set status bits (err[] output; the reference's Eigerror) ------- */
#define PL_SET_OK 0
#define PL_SET_BREAKDOWN 1  /* Lanczos restarted after an invariant subspace */
#define PL_SET_NONFINITE 2  /* NaN/Inf in the submatrix or the recurrence    */
#define PL_SET_BAD_INDEX 4  /* an index outside [0, n)                       */
#define PL_SET_BAD_K 8      /* k outside [1, PL_KMAX]                         */

/* ---- forms -------------------------------------------------------------- */
#define PL_FORM_BATCHED 0   /* persistent, binned by k, register-resident    */
#define PL_FORM_PLAIN 1     /* one set per thread block (k <= 128)           */

#define PL_KMAX 512         /* largest supported subset size                  */

int pl_version(void);                      /* 100*major + minor               */
const char *pl_status_string(int status);
int pl_last_cuda_error(void);              /* cudaError_t of the last PL_ECUDA */

/*
 * Solve every set (device pointers).
 *   A       n x n symmetric FP32 matrix, row-major, leading dimension lda >= n.
 *           Several kernels read only part of A[S,S] and mirror it (the tuned
 *           choices for 48 < k <= 192 read A[S[r]][S[c]] for r <= c; the one
 *           for 192 < k <= 256 reads the upper 32 x 32 tiles), so for an A that
 *           is not exactly symmetric the result depends on the kernel chosen
 *           for k.
 *   idx     concatenated 0-based index sets
 *   offsets NULL: uniform k, set s = idx[s*k .. s*k+k-1];
 *           else CSR (nsets+1 entries), set s = idx[offsets[s] .. offsets[s+1])
 *   form    PL_FORM_BATCHED or PL_FORM_PLAIN
 *   lmin, lmax, delta (FP64, nsets), err (int32, nsets): each nullable
 *   eig     nullable; all k eigenvalues ascending at the set's index offset
 *   det     nullable; product of the eigenvalues (FP64, nsets)
 * Per-set problems are reported in err[], not as a failed call.
 */
int pl_solve(const float *A, int n, long long lda, const int *idx, const long long *offsets,
             long long nsets, int k, int form, double *lmin, double *lmax, double *delta,
             int *err, double *eig, double *det, void *stream);

/* Allocation-free variant of pl_solve for callers that cannot call cudaMalloc
 * (a host runtime that owns the device-memory budget, code running during a
 * CUDA graph capture, plugins that must not allocate after start-up).  No
 * counterpart in the reference.  Uniform k only, 1 <= k <= 64, extremes only
 * (lambda_min, lambda_max, delta_k, err); device pointers, asynchronous on
 * `stream`.  The kernels' scratch lives in a static 32 MiB device array of the
 * library (held by every GPU that loads it until exit) instead of cudaMalloc'd
 * memory; k > 64 returns PL_ENOTSUP.  The first call on a device looks up the
 * array's device address, so make that first call before any stream capture.
 * All calls share the array: calls whose kernels overlap on the GPU race.    */
int pl_solve_noalloc(const float *A, int n, long long lda, const int *idx, long long nsets, int k,
                     double *lmin, double *lmax, double *delta, int *err, void *stream);

/* Same with HOST buffers: copies A and the sets in, solves, copies results out
 * (synchronous).  offsets/eig/det/lmin/lmax/delta/err nullable as above.
 * With uniform k, extremes only, and a k whose kernel reads each set's indices
 * one set ahead (the built-in choice for 48 < k <= 64), an idx array in pinned
 * host memory that is mapped into the device's address space (cudaMallocHost,
 * cudaHostAlloc, or registered with cudaHostRegister) is not copied: the
 * kernel reads it over the host link while it computes.  The results are the
 * same either way.                                                          */
int pl_solve_host(const float *A, int n, long long lda, const int *idx, const long long *offsets,
                  long long nsets, int k, int form, double *lmin, double *lmax, double *delta,
                  int *err, double *eig, double *det);

/* The gather alone: blocks[s*k*k + i*k + j] = A[idx[s*k+i], idx[s*k+j]] (device
 * FP32, row-major blocks), err[s] (nullable) = PL_SET_BAD_INDEX for a set with
 * an index outside [0, n).  A is symmetric (as everywhere in this library):
 * only the elements with i <= j are read, and each is written to (i, j) and
 * (j, i).  Uniform k <= PL_KMAX; asynchronous on `stream`.
 * Replaces the reference's per-thread gather LOAD_SMS4H / LOAD_SMS4HF
 * (ParaLanczos.cu:455-490), which feeds its kernels' private strips.        */
int pl_gather_blocks(const float *A, int n, long long lda, const int *idx, long long nsets, int k,
                     float *blocks, int *err, void *stream);

/* Device-side uniform-k index sets from the counter-based generator:
 * idx[s*k ..] = set (first + s) of stream `seed`, k distinct values in [0,n). */
int pl_gen_sets(unsigned long long seed, long long first, long long nsets, int n, int k, int *idx,
                void *stream);

/* Host generator of a CSR stream.  kdist: 0 fixed kmin; 1 {8,..,256} with P~1/k;
 * 2 uniform in [kmin,kmax].  With offsets == idx == NULL it only returns the
 * total index count.                                                         */
long long pl_gen_stream_host(unsigned long long seed, long long first, long long nsets, int n,
                             int kdist, int kmin, int kmax, long long *offsets, int *idx);

/* FP64 -> FP32 conversion on the device (for FP64 matrices). */
int pl_convert_f64_f32(const double *in, float *out, long long count, void *stream);

/* The drop-in entry points (calculate_subeigs*, calculate_eigs and their pl_*
 * twins) keep the caller's FP64 matrix on the device, converted to FP32, and
 * reuse it while later calls pass the same address, order and contents (a
 * 64-bit content hash of the host matrix per call); the reference uploads it
 * on every call (ParaLanczos.cu:1845-1846).  PL_DROPIN_CACHE=0 turns the
 * reuse off.  Counts of reuses (hits) and uploads (misses) on the current
 * device; either pointer may be NULL.                                        */
void pl_dropin_cache_stats(long long *hits, long long *misses);

/* ---- on-the-fly Gram form ------------------------------------------------
 * A is never materialised: each A[S,S] = Phi_S^T Phi_S is formed on the
 * tensor cores (bf16 split of the FP32 frame, FP32 accumulation, exactly
 * symmetric result) and solved like pl_solve.  Spec: the reference's Gram
 * kernels DSG_B / DSG_B1 / SG_B1 (ParaLanczos.cu:364-438, declared
 * ParaLanczos.h:24-28), which form subgrams[i*n+j] = sum_k
 * Frame[S_i + k*N] Frame[S_j + k*N] from a row-major M x N frame; no wrapper
 * of the reference calls them.  Uniform k, 1 <= k <= 128.                    */
/* Bytes of the prepared frame for an m x n Phi (m rows = Gram inner dim.).  */
long long pl_gram_prep_bytes(int m, int n);
/* Prepare the frame once: Phi is the reference's row-major m x n frame
 * (device, FP32, row stride ld >= n); prep receives pl_gram_prep_bytes bytes
 * (device, 16-byte aligned).  Asynchronous on `stream`.                      */
int pl_gram_prepare(const float *Phi, long long ld, int m, int n, void *prep, void *stream);
/* The Gram blocks themselves: blocks[s*k*k + i*k + j] = (Phi_S^T Phi_S)_ij
 * (device FP32), err[s] = PL_SET_BAD_INDEX for a set with an index outside
 * [0, n).  Each block is formed from the bf16 split and then scaled as
 * d_i d_j B_ij with d_i = sqrt(||column S_i of Phi||^2 / B_ii) (the exact
 * squared norms are part of the prepared frame), so its diagonal is exact
 * and it stays exactly symmetric.  Synchronous (returns PL_ETIMEDOUT if a
 * bounded wait gave up).                                                    */
int pl_gram_blocks(const void *prep, int m, int n, const int *idx, long long nsets, int k,
                   float *blocks, int *err, void *stream);
/* Form and solve: outputs as pl_solve (device pointers; eig at s*k).  Works
 * in chunks through a cached device buffer of at most PL_GRAM_CHUNK_MB
 * (default 2048) MiB of blocks.  Synchronous like pl_gram_blocks.           */
int pl_solve_gram(const void *prep, int m, int n, const int *idx, long long nsets, int k,
                  int form, double *lmin, double *lmax, double *delta, int *err, double *eig,
                  double *det, void *stream);

/* ---- serving: continuous batching of requests ----------------------------
 * No counterpart in the reference (each calculate_subeigs* call is one
 * synchronous batch on one matrix, ParaLanczos.cu:1725-1863).  A server keeps
 * matrices resident and solves requests (matrix, k, nsets index sets) as they
 * arrive.  The host admits queued requests in arrival order while their
 * indices fit the server's arena, uploads them and publishes a descriptor per
 * request into a ring in mapped host memory; the batching itself runs on the
 * GPU in up to `max_waves` (at most 4) device-resident request loops, one
 * CUDA graph each (a conditional WHILE node over: plan, expand, binned solve,
 * finish), requests spread over the loops by k.  Each pass a loop forms a
 * wave of about PL_SERVE_WAVE_MS (default 10) ms of GPU work -- the oldest
 * unfinished request takes up to PL_SERVE_OLDEST_SHARE (default 0.9) of it,
 * the requests with the least work left the rest, so large requests are split
 * over waves and small ones go first -- and writes results and completion
 * flags straight into mapped host memory.  A loop with no work waits at most
 * PL_SERVE_IDLE_MS (default 20) on the device and ends; the next request
 * launches it again.  `budget_bytes` bounds ALL device memory of the server
 * (loop staging and kernel scratch first, the rest is the index arena);
 * PL_EINVAL if it does not exceed the staging by at least 1 MiB.  Extremes
 * only (lambda_min, lambda_max, delta_k, err).  Host buffers; thread-safe.    */
/* `host_pool_bytes` of pinned memory stage submitted indices and results.    */
int pl_serve_create(long long budget_bytes, long long host_pool_bytes, int max_waves, void **server);
/* Register a device-resident symmetric FP32 matrix (kept by reference: it must
 * stay allocated and unchanged while the server lives).                      */
int pl_serve_add_matrix(void *server, const float *A, int n, long long lda, int *matrix_id);
/* Queue a request: idx = nsets*k host indices (copied).  PL_EBUSY: the pinned
 * pool is full (retry after collecting results); PL_EINVAL: bad arguments or a
 * request larger than the budget.                                            */
int pl_serve_submit(void *server, int matrix_id, const int *idx, long long nsets, int k,
                    long long *request_id);
/* Wait up to timeout_s for a request; on PL_OK copies its results (each
 * output nullable, nsets entries) and the submit-to-completion latency, and
 * forgets the request.  PL_ETIMEDOUT: not finished yet (still queued).       */
int pl_serve_wait(void *server, long long request_id, double timeout_s, double *lmin, double *lmax,
                  double *delta, int *err, double *latency_s);
/* out[0..15]: completed requests, sets solved, p50, p99, mean and max latency
 * (s), busy span first admission .. last completion (s), peak and total arena
 * bytes, waves formed, most loops running at once, requests queued, loop
 * launches, loops ended idle, device bytes held by the server, loops running. */
int pl_serve_stats(void *server, double *out, int nout);
int pl_serve_reset_stats(void *server);
/* Stops the loops (a wave in progress finishes first) and frees everything.  */
int pl_serve_destroy(void *server);

/* ---- ParaLanczos.h drop-ins with a status return ------------------------ */
/* Host pointers, FP64 matrix, all eigenvalues out; semantics of the named
 * reference routine (validation messages, output layout).  PL_STRICT=0 in the
 * environment lifts the reference's k <= 128 / k % 4 == 0 limits.           */
int pl_calculate_subeigs3(double *mat, int subIndexLen, int matsize, double *Eigenvalues,
                          double *Det, int *subIndex, int subn);
int pl_calculate_subeigs(double *mat, int n, double *Eigenvalues, double *Det, int *subIndex,
                         int subn);
int pl_calculate_subeigs2(double *mat, int n, int matsize, double *Eigenvalues, double *Det,
                          int *subIndex, int subn);
int pl_calculate_eigs(double *mat, int n, double *Eigenvalues, double *Det);

/* ---- the reference's kernels, launched with the caller's geometry --------
 * Launches the kernel `name` ("POS_SYM_SUBMATRIX_KER2", "POS_SYM_SUBMATRIX_KER",
 * "POS_SYM_MAT_KER", "UPPER_KER", "DSG_B", "DSG_B1" or "SG_B1": the
 * reference's ParaLanczos.h:24-36, same parameter lists) on a grid of grid_x
 * blocks of block_x x block_y threads with no dynamic shared memory -- what
 * MATLAB's CUDAKernel does with the reference's PTX (gpu_multi_subsvd2.m:
 * grid L/128, block 32; gpu_multi_subsvd.m: grid L/minor, block minor/4).
 * args: pointers to the argument values, cudaLaunchKernel's convention.
 * Device pointers; asynchronous on `stream`.  The same kernels are in
 * paralanczos_b200/ParaLanczos.ptx for MATLAB.                               */
int pl_launch_reference_kernel(const char *name, unsigned grid_x, unsigned block_x, unsigned block_y,
                               void **args, void *stream);

/* ---- tuning and measurement --------------------------------------------- */
/* Select variant `variant` of the kernel shape for bin `bin` (see
 * pl_tune_describe); -1 restores the built-in default (the autotuner's
 * choice on B200).                                                          */
int pl_tune_set(int bin, int variant);
/* The variant bin `bin` runs now (as selected by pl_tune_set or the built-in
 * default); -1 for an unknown bin.  No counterpart in the reference.        */
int pl_tune_get(int bin);
/* Writes a description of bin/variant into buf (NUL-terminated); returns the
 * number of variants of `bin`, or 0 for an unknown bin.                      */
int pl_tune_describe(int bin, int variant, char *buf, int buflen);
int pl_num_bins(void);
/* Upper k of bin b. */
int pl_bin_kmax(int bin);
/* Measured FP32 FMA throughput of this GPU (TFLOP/s), for roofline figures. */
int pl_fp32_peak(double *tflops, void *stream);
/* Measured rate of uniformly random 4-byte loads from an L2-resident array
 * (G elements/s): the ceiling of the A[S,S] gather, whose every element is
 * its own 32-byte sector.  Allocates and frees a 64 MiB buffer.              */
int pl_gather_peak(double *gelems, void *stream);
/* Releases cached device scratch, graphs and streams of this library. */
int pl_release(void);

#ifdef __cplusplus
}
#endif
#endif /* PARALANCZOS_B200_H */
