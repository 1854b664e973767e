// pl_internal.h -- host-side entry points shared between the library's
// translation units (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <mutex>

#include "pl_common.cuh"

namespace pl {

// One uniform-k launch of the batched (or plain) Lanczos kernels on M.
int api_solve_uniform(const MatrixF32& M, const int* idx, long long nsets, int k, int form,
                      const SetOutputs& out, cudaStream_t st);

// Number of k bins of the batched kernels.
int api_num_bins();

// Device scratch (bytes) of one api_launch_binned call over nsets sets.
size_t api_binned_scratch(long long nsets, int form, bool all);

// Binned CSR launch enqueued directly on `st` (no graph capture): device-side
// counting sort of the sets by k bin, then one persistent kernel per bin on
// the side streams side[0..nbins) (fork/join through the given events).
// `scratch` holds api_binned_scratch(nsets, ...) bytes used by this launch
// alone until it completes.  With nsets_dev non-null the set count is read
// on the device when the launch runs (nsets is then its upper bound), so the
// same enqueued work can be captured once and replayed for changing counts.
int api_launch_binned(const MatrixF32& M, const int* idx, const long long* offsets, long long nsets,
                      int form, const SetOutputs& out, void* scratch, cudaStream_t st,
                      const cudaStream_t* side, cudaEvent_t fork, const cudaEvent_t* join,
                      const long long* nsets_dev = nullptr);

// Loads the binned launch's kernels of `form` and caches their launch
// attributes, so that api_launch_binned can then run inside a stream capture.
int api_prepare_binned(int form, bool all);

// Serialises calls that touch the per-device cached state.
std::mutex& api_mutex();

// Records the CUDA error returned by pl_last_cuda_error().
void api_note_cuda(cudaError_t e);

// Multiprocessors of the current device.
int api_device_sms();

// Frees the Gram form's cached device buffers (called by pl_release).
void gram_release();

// The drop-in entry points' solve of nsets uniform-k sets of an FP64 host
// matrix (n x n): the matrix is cached on the device (FP32) between calls with
// the same address, order and contents; all k eigenvalues, det and err out.
int api_solve_f64_host(const double* mat, int n, const int* subIndex, long long nsets, int k, int form,
                       double* eig, double* det, int* err);

// Hits and misses of the drop-in matrix cache on the current device.
void api_dropin_cache_stats(long long* hits, long long* misses);

}  // namespace pl
