// pl_sync.cuh -- shared-memory mbarrier helpers with bounded waits.
//
// Every wait on an mbarrier is bounded by %globaltimer (2 s): a wait that
// gives up sets the CTA's abort flag and, where given, a device status word,
// so a kernel whose partner role stopped making progress returns instead of
// spinning.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pl {

constexpr unsigned long long kWaitNs = 2000000000ull;  // bounded waits: 2 s

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Arrive with release semantics (the default of mbarrier.arrive).
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase with the given parity.  false: gave up (timeout
// here, or another role already aborted); the abort flag is then set and, if
// status is given, *status = 1.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort,
                                          int* status) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try(bar, parity)) return true;
    if ((i & 31) == 0) {
      if (*abort) return false;
      if (globaltimer() - t0 > kWaitNs) {
        *abort = 1;
        if (status) atomicExch(status, 1);
        return false;
      }
    }
  }
}

}  // namespace pl
