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

// Serialises calls that touch the per-device cached state.
std::mutex& api_mutex();

// Records the CUDA error returned by pl_last_cuda_error().
void api_note_cuda(cudaError_t e);

// Multiprocessors of the current device.
int api_device_sms();

// Frees the Gram form's cached device buffers (called by pl_release).
void gram_release();

}  // namespace pl
