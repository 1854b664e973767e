// pl_api.cu -- host dispatch and the C ABI of libparalanczos_b200.so.
//
// Replaces the host API of the reference (ParaLanczos.cu:1642-1863, declared in
// ParaLanczos.h:39-47).  Differences: no cudaDeviceReset, device scratch is
// cached per device, results and per-set status are returned, nothing is
// printed unless PL_VERBOSE=1 (then the reference's stdout lines are
// reproduced), and uneven k is binned on the device and run from a captured
// CUDA graph.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/paralanczos.h"
#include "pl_internal.h"
#include "pl_kernels.cuh"

using namespace pl;

namespace {

thread_local int g_last_cuda = 0;
std::mutex g_mu;

#define PL_CU(call)                              \
  do {                                           \
    cudaError_t e_ = (call);                     \
    if (e_ != cudaSuccess) {                     \
      g_last_cuda = (int)e_;                     \
      return e_ == cudaErrorMemoryAllocation ? PL_ENOMEM : PL_ECUDA; \
    }                                            \
  } while (0)

int device_sms() {
  static int sms[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return 148;
  if (!sms[dev]) cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev);
  return sms[dev] > 0 ? sms[dev] : 148;
}

// nitems < 0: the item count lives on the device.  prep: only load the kernel
// and cache its launch attributes (done before a stream capture starts).
// PL_VERBOSE=2 logs launch configurations to stderr.
int verbosity() {
  static int v = [] {
    const char* e = getenv("PL_VERBOSE");
    return e ? atoi(e) : 0;
  }();
  return v;
}

typedef cudaError_t (*LaunchFn)(const MatrixF32&, const SetSource&, const SetOutputs&, long long,
                                void*, cudaStream_t, bool prep);
// Bytes of device scratch a variant needs at its full (persistent) grid.
typedef size_t (*ScratchFn)();

template <class K>
int occupancy(K kern, int cta, size_t dsmem) {
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, cta, dsmem);
  return occ > 0 ? occ : 1;
}

long long grid_for(long long nitems, int per_cta, int occ) {
  const long long full = (long long)device_sms() * occ;
  if (nitems < 0) return full;  // count lives on the device
  const long long need = (nitems + per_cta - 1) / per_cta;
  return need < full ? (need > 0 ? need : 1) : full;
}

template <int KB, int RPT, int TPR, int CTA, int MINB, bool ALL>
cudaError_t launch_reg(const MatrixF32& M, const SetSource& src, const SetOutputs& out,
                       long long nitems, void* scratch, cudaStream_t st, bool prep) {
  auto kern = k_reg_solve<KB, RPT, TPR, CTA, MINB, ALL>;
  static int occ = occupancy(kern, CTA, 0);
  if (prep) {
    cudaFuncAttributes fa;
    return cudaFuncGetAttributes(&fa, kern);
  }
  constexpr int GPC = CTA / Cfg<KB, RPT, TPR>::NT;
  const long long grid = grid_for(nitems, GPC, occ);
  kern<<<(unsigned)grid, CTA, 0, st>>>(M, src, out, (double2*)scratch);
  return cudaGetLastError();
}

// Queue buffer of the deferred bisection: per group Q = NT/2 tridiagonals of KB.
template <int KB, int RPT, int TPR, int CTA, int MINB, bool ALL>
size_t scratch_reg() {
  if (ALL) return 0;
  auto kern = k_reg_solve<KB, RPT, TPR, CTA, MINB, ALL>;
  constexpr int NT = Cfg<KB, RPT, TPR>::NT;
  const size_t grid = (size_t)device_sms() * occupancy(kern, CTA, 0);
  return grid * (CTA / NT) * (NT / 2) * KB * sizeof(double2);
}

template <int KB, int RPT, int CTA, int MINB, bool ALL>
cudaError_t launch_sa(const MatrixF32& M, const SetSource& src, const SetOutputs& out,
                      long long nitems, void* scratch, cudaStream_t st, bool prep) {
  auto kern = k_sa_solve<KB, RPT, CTA, MINB, ALL>;
  constexpr int GPC = CTA / CfgSA<KB, RPT>::NT;
  const size_t dsm = sizeof(SASmem<KB, RPT>) * GPC;
  static int occ = [&] {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm);
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    return occupancy(kern, CTA, dsm);
  }();
  if (prep) {
    cudaFuncAttributes fa;
    return cudaFuncGetAttributes(&fa, kern);
  }
  const long long grid = grid_for(nitems, GPC, occ);
  kern<<<(unsigned)grid, CTA, dsm, st>>>(M, src, out, (double2*)scratch);
  return cudaGetLastError();
}

template <int KB, int RPT, int CTA, int MINB, bool ALL>
size_t scratch_sa() {
  if (ALL) return 0;
  auto kern = k_sa_solve<KB, RPT, CTA, MINB, ALL>;
  constexpr int NT = CfgSA<KB, RPT>::NT;
  const size_t dsm = sizeof(SASmem<KB, RPT>) * (CTA / NT);
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm);
  cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  const size_t grid = (size_t)device_sms() * occupancy(kern, CTA, dsm);
  return grid * (CTA / NT) * (NT / 2) * KB * sizeof(double2);
}

template <int KB, int RPT, int CTA, int REGS, bool ALL>
cudaError_t launch_sar(const MatrixF32& M, const SetSource& src, const SetOutputs& out,
                       long long nitems, void* scratch, cudaStream_t st, bool prep) {
  auto kern = k_sa_solve_r<KB, RPT, CTA, REGS, ALL>;
  constexpr int GPC = CTA / CfgSA<KB, RPT>::NT;
  const size_t dsm = sizeof(SASmem<KB, RPT>) * GPC;
  static int occ = [&] {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm);
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    return occupancy(kern, CTA, dsm);
  }();
  if (prep) {
    cudaFuncAttributes fa;
    return cudaFuncGetAttributes(&fa, kern);
  }
  const long long grid = grid_for(nitems, GPC, occ);
  kern<<<(unsigned)grid, CTA, dsm, st>>>(M, src, out, (double2*)scratch);
  return cudaGetLastError();
}

template <int KB, int RPT, int CTA, int REGS, bool ALL>
size_t scratch_sar() {
  if (ALL) return 0;
  auto kern = k_sa_solve_r<KB, RPT, CTA, REGS, ALL>;
  constexpr int NT = CfgSA<KB, RPT>::NT;
  const size_t dsm = sizeof(SASmem<KB, RPT>) * (CTA / NT);
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm);
  cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  const size_t grid = (size_t)device_sms() * occupancy(kern, CTA, dsm);
  return grid * (CTA / NT) * (NT / 2) * KB * sizeof(double2);
}

// shared-A with the next set's triangle prefetched (extremes mode); AR float4
// chunks of each row of A_S in registers
template <int KB, int RPT, int CTA, int REGS, int AR = 0>
cudaError_t launch_sap(const MatrixF32& M, const SetSource& src, const SetOutputs& out, long long nitems,
                       void* scratch, cudaStream_t st, bool prep) {
  auto kern = k_sa_solve_p<KB, RPT, CTA, REGS, AR>;
  constexpr int GPC = CTA / CfgSA<KB, RPT>::NT;
  const size_t dsm = (sizeof(SASmem<KB, RPT>) + sizeof(SAStage<KB, CfgSA<KB, RPT>::NT>)) * GPC;
  static int occ = [&] {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm);
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    return occupancy(kern, CTA, dsm);
  }();
  if (prep) {
    cudaFuncAttributes fa;
    return cudaFuncGetAttributes(&fa, kern);
  }
  const long long grid = grid_for(nitems, GPC, occ);
  kern<<<(unsigned)grid, CTA, dsm, st>>>(M, src, out, (double2*)scratch);
  return cudaGetLastError();
}

template <int KB, int RPT, int CTA, int REGS, int AR = 0>
size_t scratch_sap() {
  auto kern = k_sa_solve_p<KB, RPT, CTA, REGS, AR>;
  constexpr int NT = CfgSA<KB, RPT>::NT;
  const size_t dsm = (sizeof(SASmem<KB, RPT>) + sizeof(SAStage<KB, CfgSA<KB, RPT>::NT>)) * (CTA / NT);
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm);
  cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  const size_t grid = (size_t)device_sms() * occupancy(kern, CTA, dsm);
  return grid * (CTA / NT) * (NT / 2) * KB * sizeof(double2);
}

template <int KB, int CTA, int MINB>
cudaError_t launch_sa2(const MatrixF32& M, const SetSource& src, const SetOutputs& out,
                       long long nitems, void* scratch, cudaStream_t st, bool prep) {
  auto kern = k_sa2_solve<KB, CTA, MINB>;
  constexpr int GPC = CTA / CfgSA2<KB>::NT;
  const size_t dsm = sizeof(SA2Smem<KB>) * GPC;
  static int occ = [&] {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm);
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    return occupancy(kern, CTA, dsm);
  }();
  if (prep) {
    cudaFuncAttributes fa;
    return cudaFuncGetAttributes(&fa, kern);
  }
  const long long grid = grid_for(nitems, GPC, occ);
  kern<<<(unsigned)grid, CTA, dsm, st>>>(M, src, out, (double2*)scratch);
  return cudaGetLastError();
}

template <int KB, int CTA, int MINB>
size_t scratch_sa2() {
  auto kern = k_sa2_solve<KB, CTA, MINB>;
  constexpr int NT = CfgSA2<KB>::NT;
  const size_t dsm = sizeof(SA2Smem<KB>) * (CTA / NT);
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm);
  cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  const size_t grid = (size_t)device_sms() * occupancy(kern, CTA, dsm);
  return grid * (CTA / NT) * (NT / 2) * KB * sizeof(double2);
}

template <int KB, bool ALL>
cudaError_t launch_plain(const MatrixF32& M, const SetSource& src, const SetOutputs& out,
                         long long nitems, void*, cudaStream_t st, bool prep) {
  constexpr int NT = KB < 32 ? 32 : KB;
  const size_t dsm = sizeof(float) * 2 * KB * (KB + 1);
  auto kern = k_plain<KB, ALL>;
  static bool attr = [&] {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm);
    return true;
  }();
  (void)attr;
  if (prep) {
    cudaFuncAttributes fa;
    return cudaFuncGetAttributes(&fa, kern);
  }
  // one set per thread block; grid-stride only beyond the grid limit
  long long grid = nitems < 0 ? (long long)device_sms() * 16 : nitems;
  if (grid > 0x7fffffffLL) grid = 0x7fffffffLL;
  if (grid < 1) grid = 1;
  kern<<<(unsigned)grid, NT, dsm, st>>>(M, src, out);
  return cudaGetLastError();
}

template <int KM, bool ALL>
cudaError_t launch_large(const MatrixF32& M, const SetSource& src, const SetOutputs& out,
                         long long nitems, void* scratch, cudaStream_t st, bool prep) {
  auto kern = k_large<KM, ALL>;
  if (prep) {
    cudaFuncAttributes fa;
    return cudaFuncGetAttributes(&fa, kern);
  }
  const long long grid = grid_for(nitems, 1, 1);
  kern<<<(unsigned)grid, 256, 0, st>>>(M, src, out, (float*)scratch);
  return cudaGetLastError();
}

template <int KB, int CS, int NTC, int RPT = 1>
cudaError_t launch_cluster(const MatrixF32& M, const SetSource& src, const SetOutputs& out,
                           long long nitems, void*, cudaStream_t st, bool prep) {
  auto kern = k_cluster_solve<KB, CS, NTC, RPT>;
  const size_t dsm = sizeof(ClusterSmem<KB, CS, NTC>);
  static int maxcl = [&] {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm);
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CS * 64, 1, 1);
    cfg.blockDim = dim3(NTC, 1, 1);
    cfg.dynamicSmemBytes = dsm;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess || n < 1) {
      cudaGetLastError();
      n = device_sms() / CS;
    }
    return n;
  }();
  if (prep) {
    cudaFuncAttributes fa;
    return cudaFuncGetAttributes(&fa, kern);
  }
  long long ncl = maxcl;
  if (nitems >= 0 && nitems < ncl) ncl = nitems > 0 ? nitems : 1;
  if (verbosity() >= 2)
    fprintf(stderr, "paralanczos: cluster KB=%d CS=%d NTC=%d: %lld clusters (max resident %d), %zu B smem/CTA\n",
            KB, CS, NTC, ncl, maxcl, dsm);
  kern<<<(unsigned)(ncl * CS), NTC, dsm, st>>>(M, src, out);
  return cudaGetLastError();
}

template <int NB, int NW, int TPW, int MINB>
cudaError_t launch_sym(const MatrixF32& M, const SetSource& src, const SetOutputs& out, long long nitems,
                       void*, cudaStream_t st, bool prep) {
  auto kern = k_sym_solve<NB, NW, TPW, MINB>;
  const size_t dsm = sizeof(SymSmem<NB, NW>);
  static int occ = [&] {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm);
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    return occupancy(kern, NW * 32, dsm);
  }();
  if (prep) {
    cudaFuncAttributes fa;
    return cudaFuncGetAttributes(&fa, kern);
  }
  const long long grid = grid_for(nitems, 1, occ);
  if (verbosity() >= 2)
    fprintf(stderr, "paralanczos: sym NB=%d NW=%d TPW=%d: %lld CTAs (%d per SM), %zu B smem/CTA\n", NB, NW, TPW,
            grid, occ, dsm);
  kern<<<(unsigned)grid, NW * 32, dsm, st>>>(M, src, out);
  return cudaGetLastError();
}

template <int KM>
size_t scratch_large() {
  return sizeof(float) * 2 * (size_t)KM * KM * (size_t)device_sms();
}
size_t scratch_none() { return 0; }

struct Variant {
  const char* desc;
  LaunchFn fn[2];       // [extremes only, all eigenvalues]
  ScratchFn scratch[2]; // device scratch at the full grid
  // (extremes mode) each group reads its next set's indices one set ahead,
  // so their latency is hidden behind a whole set's Lanczos steps
  bool indices_ahead;
};

#define REG(KB, RPT, TPR, CTA, MINB)                                                          \
  Variant {                                                                                    \
    "reg KB=" #KB " RPT=" #RPT " TPR=" #TPR " CTA=" #CTA " MINB=" #MINB,                       \
        {launch_reg<KB, RPT, TPR, CTA, MINB, false>, launch_reg<KB, RPT, TPR, CTA, MINB, true>}, \
        {scratch_reg<KB, RPT, TPR, CTA, MINB, false>, scratch_none}                            \
  }
#define SA(KB, RPT, CTA, MINB)                                                               \
  Variant {                                                                                    \
    "sharedA KB=" #KB " RPT=" #RPT " CTA=" #CTA " MINB=" #MINB,                                \
        {launch_sa<KB, RPT, CTA, MINB, false>, launch_sa<KB, RPT, CTA, MINB, true>},          \
        {scratch_sa<KB, RPT, CTA, MINB, false>, scratch_none}                                  \
  }
#define SAR(KB, RPT, CTA, REGS)                                                              \
  Variant {                                                                                    \
    "sharedA KB=" #KB " RPT=" #RPT " CTA=" #CTA " REGS=" #REGS,                                \
        {launch_sar<KB, RPT, CTA, REGS, false>, launch_sar<KB, RPT, CTA, REGS, true>},        \
        {scratch_sar<KB, RPT, CTA, REGS, false>, scratch_none}                                 \
  }
// the next set's upper triangle prefetched into shared memory during this set's steps
#define SAP(KB, RPT, CTA, REGS)                                                              \
  Variant {                                                                                    \
    "sharedA prefetch KB=" #KB " RPT=" #RPT " CTA=" #CTA " REGS=" #REGS,                       \
        {launch_sap<KB, RPT, CTA, REGS>, nullptr}, {scratch_sap<KB, RPT, CTA, REGS>, scratch_none}, \
        true                                                                                     \
  }
#define SAPR(KB, RPT, CTA, REGS, AR)                                                         \
  Variant {                                                                                    \
    "sharedA prefetch KB=" #KB " RPT=" #RPT " CTA=" #CTA " REGS=" #REGS " AREG=" #AR,          \
        {launch_sap<KB, RPT, CTA, REGS, AR>, nullptr},                                          \
        {scratch_sap<KB, RPT, CTA, REGS, AR>, scratch_none}, true                               \
  }
#define SA2(KB, CTA, MINB)                                                                   \
  Variant {                                                                                    \
    "sharedA 2 threads/row KB=" #KB " CTA=" #CTA " MINB=" #MINB,                               \
        {launch_sa2<KB, CTA, MINB>, nullptr}, {scratch_sa2<KB, CTA, MINB>, scratch_none}       \
  }
#define CLUSTER(KB, CS, NTC)                                                                  \
  Variant {                                                                                     \
    "cluster KB=" #KB " CS=" #CS " NTC=" #NTC,                                                  \
        {launch_cluster<KB, CS, NTC>, nullptr}, {scratch_none, scratch_none}                    \
  }
// RPT rows per thread (each with KB / TPR columns of P)
#define CLUSTERR(KB, CS, NTC, RPT)                                                            \
  Variant {                                                                                     \
    "cluster KB=" #KB " CS=" #CS " NTC=" #NTC " RPT=" #RPT,                                     \
        {launch_cluster<KB, CS, NTC, RPT>, nullptr}, {scratch_none, scratch_none}               \
  }
// upper 32 x 32 tiles of A_S and P, one set per CTA (NB blocks of 32, NW warps of TPW tiles)
#define SYM(NB, NW, TPW, MINB)                                                                 \
  Variant {                                                                                      \
    "sym NB=" #NB " NW=" #NW " TPW=" #TPW " MINB=" #MINB,                                        \
        {launch_sym<NB, NW, TPW, MINB>, nullptr}, {scratch_none, scratch_none}                   \
  }
#define LARGE(KM) \
  Variant {                                                                             \
    "large KM=" #KM " CTA=256", {launch_large<KM, false>, launch_large<KM, true>},      \
        {scratch_large<KM>, scratch_large<KM>}                                           \
  }

const int kBinK[] = {8, 16, 32, 48, 64, 96, 128, 192, 256, 384, 512};
constexpr int kNumBins = 11;

const std::vector<Variant>& variants(int b) {
  static const std::vector<Variant> v[kNumBins] = {
      {REG(8, 2, 1, 128, 4), REG(8, 1, 1, 128, 4), SA(8, 2, 128, 4)},
      {REG(16, 2, 1, 128, 4), REG(16, 1, 1, 128, 4), SA(16, 2, 128, 4)},
      {REG(32, 2, 1, 128, 3), REG(32, 1, 1, 128, 4), SA(32, 2, 128, 4), SAP(32, 2, 128, 128)},
      {SA(48, 3, 128, 2), REG(48, 3, 2, 128, 2)},
      {REG(64, 1, 1, 128, 3), SA(64, 2, 128, 3), REG(64, 1, 1, 128, 2), SA(64, 2, 128, 2),
       SAR(64, 2, 96, 224), SAR(64, 2, 128, 224), SAR(64, 2, 64, 200), SAP(64, 2, 128, 224),
       SAP(64, 2, 64, 224), SAP(64, 2, 96, 224), SAPR(64, 2, 128, 255, 4), SAPR(64, 2, 64, 255, 4)},
      {SA(96, 1, 96, 3), SA2(96, 96, 3), SA2(96, 96, 4), SA(96, 1, 96, 4)},
      {SA(128, 1, 128, 3), REG(128, 1, 2, 256, 1), SA(128, 1, 128, 2), SA2(128, 128, 2), SYM(4, 5, 2, 3),
       SYM(4, 10, 1, 2)},
      {CLUSTER(192, 2, 384), LARGE(256), CLUSTER(192, 4, 192), CLUSTER(192, 1, 384), CLUSTER(192, 1, 768),
       CLUSTERR(192, 1, 384, 2), CLUSTERR(192, 1, 384, 4), SYM(6, 11, 2, 1), SYM(6, 21, 1, 1),
       SYM(6, 16, 2, 1)},
      {CLUSTER(256, 2, 512), LARGE(256), CLUSTER(256, 4, 256), CLUSTER(256, 8, 256), CLUSTER(256, 2, 256),
       CLUSTERR(256, 2, 256, 2), CLUSTERR(256, 2, 256, 4), SYM(8, 12, 3, 1)},
      {CLUSTER(384, 4, 384), LARGE(512), CLUSTER(384, 8, 192), CLUSTER(384, 6, 256), CLUSTERR(384, 6, 256, 2),
       CLUSTERR(384, 6, 256, 4), CLUSTERR(384, 4, 384, 4)},
      {CLUSTER(512, 8, 256), LARGE(512), CLUSTER(512, 8, 512), CLUSTERR(512, 8, 256, 2),
       CLUSTERR(512, 8, 256, 4)},
  };
  return v[b];
}

// Built-in shape per bin: the autotuner's choices on B200 (tuning.json), so a
// caller that never runs the Python tuner (a C program, MATLAB) gets them too.
const int kDefaultVariant[kNumBins] = {0, 0, 2, 1, 10, 1, 3, 6, 7, 6, 3};
int g_variant[kNumBins] = {0, 0, 2, 1, 10, 1, 3, 6, 7, 6, 3};

int bin_of_k(int k) {
  for (int b = 0; b < kNumBins; ++b)
    if (k <= kBinK[b]) return b;
  return -1;
}

const Variant& chosen(int b) {
  const auto& v = variants(b);
  int i = g_variant[b];
  if (i < 0 || i >= (int)v.size()) i = 0;
  return v[i];
}

// The chosen variant if it implements the requested mode (extremes / all
// eigenvalues), else the first variant of the bin that does.
const Variant& chosen_for(int b, bool all) {
  const Variant& v = chosen(b);
  if (v.fn[all ? 1 : 0]) return v;
  for (const Variant& w : variants(b))
    if (w.fn[all ? 1 : 0]) return w;
  return v;
}

// Plain form kernels by k bin (k <= 128).
LaunchFn plain_fn(int k, bool all) {
  if (k <= 16) return all ? launch_plain<16, true> : launch_plain<16, false>;
  if (k <= 32) return all ? launch_plain<32, true> : launch_plain<32, false>;
  if (k <= 64) return all ? launch_plain<64, true> : launch_plain<64, false>;
  if (k <= 128) return all ? launch_plain<128, true> : launch_plain<128, false>;
  return nullptr;
}

// ----------------------------------------------------------------------------
// Per-device cached scratch (grow-only).
// ----------------------------------------------------------------------------
struct DevScratch {
  void* p = nullptr;
  size_t bytes = 0;
};

// The drop-in entry points' matrix, cached on the device between calls: the
// caller's FP64 host matrix identified by its address, order and a content
// hash, converted to FP32 on the device.
struct MatCache {
  const double* host = nullptr;
  int n = 0;
  uint64_t hash = 0;
  bool valid = false;
  long long hits = 0, misses = 0;
};

struct DevState {
  DevScratch large;    // k_large slots
  DevScratch bins;     // counts / starts / cursor / perm
  DevScratch upload;   // pl_solve_host and drop-in staging
  DevScratch mat64;    // drop-in: the FP64 matrix as uploaded
  DevScratch mat32;    // drop-in: its FP32 conversion (MatCache)
  MatCache mc;
  cudaStream_t side[kNumBins] = {};
  cudaStream_t cap = nullptr;  // private stream the CSR graph is captured on
  cudaEvent_t ev_fork = nullptr;
  cudaEvent_t ev_join[kNumBins] = {};
  struct GraphEntry {
    cudaGraphExec_t exec;
  };
  std::unordered_map<std::string, GraphEntry> graphs;
};

DevState g_state[64];

DevState& state() {
  int dev = 0;
  cudaGetDevice(&dev);
  return g_state[dev < 0 || dev >= 64 ? 0 : dev];
}

void drop_graphs(DevState& d) {
  for (auto& kv : d.graphs) cudaGraphExecDestroy(kv.second.exec);
  d.graphs.clear();
}

// Grow-only scratch.  A reallocation invalidates every cached graph of the
// device (they hold pointers into the scratch buffers).
int ensure(DevScratch& s, size_t bytes) {
  if (s.bytes >= bytes) return PL_OK;
  DevState& d = state();
  if (s.p) {
    cudaDeviceSynchronize();
    drop_graphs(d);
    cudaFree(s.p);
    s.p = nullptr;
    s.bytes = 0;
  }
  PL_CU(cudaMalloc(&s.p, bytes));
  s.bytes = bytes;
  return PL_OK;
}

int ensure_streams(DevState& d) {
  if (d.ev_fork) return PL_OK;
  PL_CU(cudaEventCreateWithFlags(&d.ev_fork, cudaEventDisableTiming));
  PL_CU(cudaStreamCreateWithFlags(&d.cap, cudaStreamNonBlocking));
  for (int b = 0; b < kNumBins; ++b) {
    PL_CU(cudaStreamCreateWithFlags(&d.side[b], cudaStreamNonBlocking));
    PL_CU(cudaEventCreateWithFlags(&d.ev_join[b], cudaEventDisableTiming));
  }
  return PL_OK;
}

bool env_flag(const char* name, bool dflt) {
  const char* v = getenv(name);
  if (!v || !*v) return dflt;
  return !(v[0] == '0' || v[0] == 'n' || v[0] == 'N' || v[0] == 'f' || v[0] == 'F');
}

// Uniform k: one kernel.
int solve_uniform(const MatrixF32& M, const int* idx, long long nsets, int k, int form,
                  const SetOutputs& out, cudaStream_t st) {
  const bool all = out.eig || out.det;
  SetSource src{idx, nullptr, k, nullptr, nullptr, nullptr, nsets};
  if (form == PL_FORM_PLAIN && k <= 128) {
    PL_CU(plain_fn(k, all)(M, src, out, nsets, nullptr, st, false));
    return PL_OK;
  }
  const int b = bin_of_k(k);
  if (b < 0) return PL_ENOTSUP;
  const Variant& v = chosen_for(b, all);
  void* scratch = nullptr;
  const size_t need = v.scratch[all ? 1 : 0]();
  if (need) {
    int rc = ensure(state().large, need);
    if (rc) return rc;
    scratch = state().large.p;
  }
  PL_CU(v.fn[all ? 1 : 0](M, src, out, nsets, scratch, st, false));
  return PL_OK;
}

// Per-bin queue-scratch layout of one binned launch: region b at off[b].
size_t binned_qscratch(int form, bool all, size_t off[kNumBins]) {
  size_t total = 0;
  for (int b = 0; b < kNumBins; ++b) {
    off[b] = total;
    const bool plain_bin = form == PL_FORM_PLAIN && kBinK[b] <= 128;
    const size_t need = plain_bin ? 0 : chosen_for(b, all).scratch[all ? 1 : 0]();
    total += (need + 255) & ~(size_t)255;
  }
  return total;
}

void binned_fns(int form, bool all, LaunchFn fns[kNumBins]) {
  for (int b = 0; b < kNumBins; ++b)
    fns[b] = (form == PL_FORM_PLAIN && kBinK[b] <= 128) ? plain_fn(kBinK[b], all)
                                                        : chosen_for(b, all).fn[all ? 1 : 0];
}

// The binned sequence on stream cs: count sets per k bin, scan, scatter the
// set ids into per-bin queues (perm), flag bad k, then one persistent launch
// per bin on the forked side streams (largest k first, so the small-k kernels
// fill the tail), joined back into cs.  hdr: 48 ints (counts, starts, cursor)
// followed by nsets ints of perm.
cudaError_t enqueue_binned(const MatrixF32& M, const int* idx, const long long* offsets,
                           long long nsets, const SetOutputs& out, const LaunchFn fns[kNumBins],
                           int* hdr, char* qscratch, const size_t qoff[kNumBins], cudaStream_t cs,
                           const cudaStream_t side[kNumBins], cudaEvent_t fork,
                           const cudaEvent_t join[kNumBins], const long long* nsets_dev = nullptr) {
  const int nb = kNumBins;
  int* counts = hdr;
  int* starts = hdr + 16;
  int* cursor = hdr + 32;
  int* perm = hdr + 48;
  BinTable bt;
  bt.nb = nb;
  for (int b = 0; b < nb; ++b) bt.kmax[b] = kBinK[b];
  cudaError_t e = cudaSuccess;
  auto note = [&](cudaError_t x) {
    if (e == cudaSuccess && x != cudaSuccess) e = x;
  };
  note(cudaMemsetAsync(counts, 0, sizeof(int) * 16, cs));
  const int tb = 256;
  const long long g = (nsets + tb - 1) / tb;
  const unsigned grid = (unsigned)(g < 4096 ? (g > 0 ? g : 1) : 4096);
  k_bin_count<<<grid, tb, 0, cs>>>(offsets, nsets, bt, counts, nsets_dev);
  note(cudaGetLastError());
  k_bin_scan<<<1, 32, 0, cs>>>(counts, nb, starts, cursor);
  note(cudaGetLastError());
  k_bin_scatter<<<grid, tb, 0, cs>>>(offsets, nsets, bt, starts, cursor, perm, nsets_dev);
  note(cudaGetLastError());
  k_mark_bad_k<<<64, 256, 0, cs>>>(perm, starts + nb, counts + nb, offsets, out);
  note(cudaGetLastError());
  note(cudaEventRecord(fork, cs));
  for (int b = nb - 1; b >= 0 && e == cudaSuccess; --b) {
    note(cudaStreamWaitEvent(side[b], fork, 0));
    SetSource src{idx, offsets, 0, perm, starts + b, counts + b, 0};
    note(fns[b](M, src, out, -1, qscratch + qoff[b], side[b], false));
    note(cudaEventRecord(join[b], side[b]));
    note(cudaStreamWaitEvent(cs, join[b], 0));
  }
  return e;
}

// Uneven k (CSR): device binning, then one persistent launch per non-empty
// bin on forked streams, all captured into one CUDA graph (cached by the call
// signature) and launched as one unit.
int solve_csr(const MatrixF32& M, const int* idx, const long long* offsets, long long nsets,
              int form, const SetOutputs& out, cudaStream_t st) {
  const bool all = out.eig || out.det;
  DevState& d = state();
  int rc = ensure_streams(d);
  if (rc) return rc;
  rc = ensure(d.bins, sizeof(int) * (48 + (size_t)nsets));
  if (rc) return rc;
  // every bin gets its own scratch region: the bins run concurrently
  size_t qoff[kNumBins];
  const size_t qtotal = binned_qscratch(form, all, qoff);
  rc = ensure(d.large, qtotal > 0 ? qtotal : 256);
  if (rc) return rc;
  char keybuf[512];
  int kl = snprintf(keybuf, sizeof keybuf, "%p|%d|%lld|%p|%p|%lld|%d|%p|%p|%p|%p|%p|%p|", (const void*)M.A, M.n,
                    M.lda, (const void*)idx, (const void*)offsets, nsets, form, (void*)out.lmin,
                    (void*)out.lmax, (void*)out.delta, (void*)out.err, (void*)out.eig, (void*)out.det);
  for (int b = 0; b < kNumBins && kl > 0 && kl < (int)sizeof keybuf - 4; ++b)
    kl += snprintf(keybuf + kl, sizeof keybuf - (size_t)kl, "%d,", g_variant[b]);
  const std::string key(keybuf);
  auto it = d.graphs.find(key);
  if (it == d.graphs.end()) {
    LaunchFn fns[kNumBins];
    binned_fns(form, all, fns);
    // load every kernel before the capture: nothing that may load a module
    // or set a function attribute runs while the stream is capturing
    for (int b = 0; b < kNumBins; ++b) PL_CU(fns[b](M, SetSource{}, out, 0, nullptr, d.side[b], true));
    cudaStream_t cs = d.cap;  // graphs do not depend on the stream they were captured on
    PL_CU(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue_binned(M, idx, offsets, nsets, out, fns, (int*)d.bins.p, (char*)d.large.p,
                                   qoff, cs, d.side, d.ev_fork, d.ev_join);
    cudaGraph_t graph = nullptr;
    {
      cudaError_t e2 = cudaStreamEndCapture(cs, &graph);  // always ends the capture
      if (e == cudaSuccess) e = e2;
    }
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      if (exec) cudaGraphExecDestroy(exec);
      cudaGetLastError();
      g_last_cuda = (int)e;
      return PL_ECUDA;
    }
    it = d.graphs.emplace(key, DevState::GraphEntry{exec}).first;
  }
  PL_CU(cudaGraphLaunch(it->second.exec, st));
  return PL_OK;
}

int validate_common(const float* A, int n, long long lda, const int* idx, long long nsets, int k,
                    const long long* offsets, int form) {
  if (nsets < 0 || n <= 0 || lda < n) return PL_EINVAL;
  if (nsets == 0) return PL_OK;
  if (!A || !idx) return PL_EINVAL;
  if (form != PL_FORM_BATCHED && form != PL_FORM_PLAIN) return PL_EINVAL;
  if (!offsets) {
    if (k < 1) return PL_EINVAL;
    if (k > PL_KMAX) return PL_ENOTSUP;
    if (k > n) return PL_EINVAL;
  }
  return PL_OK;
}

int solve_dev(const float* A, int n, long long lda, const int* idx, const long long* offsets,
              long long nsets, int k, int form, const SetOutputs& out, cudaStream_t st) {
  int rc = validate_common(A, n, lda, idx, nsets, k, offsets, form);
  if (rc || nsets == 0) return rc;
  MatrixF32 M{A, lda, n};
  if (!offsets) return solve_uniform(M, idx, nsets, k, form, out, st);
  return solve_csr(M, idx, offsets, nsets, form, out, st);
}

// Staging for host-buffer calls: one grow-only device buffer carved in place.
struct Carve {
  char* base;
  size_t off;
  template <class T>
  T* take(size_t count) {
    off = (off + 255) & ~(size_t)255;
    T* p = (T*)(base + off);
    off += sizeof(T) * count;
    return p;
  }
};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

namespace pl {
int api_solve_uniform(const MatrixF32& M, const int* idx, long long nsets, int k, int form,
                      const SetOutputs& out, cudaStream_t st) {
  return solve_uniform(M, idx, nsets, k, form, out, st);
}
std::mutex& api_mutex() { return g_mu; }
int api_num_bins() { return kNumBins; }
size_t api_binned_scratch(long long nsets, int form, bool all) {
  size_t qoff[kNumBins];
  return align256(sizeof(int) * (48 + (size_t)nsets)) + binned_qscratch(form, all, qoff);
}
int api_prepare_binned(int form, bool all) {
  LaunchFn fns[kNumBins];
  binned_fns(form, all, fns);
  SetOutputs out{};
  for (int b = 0; b < kNumBins; ++b) PL_CU(fns[b](MatrixF32{}, SetSource{}, out, 0, nullptr, 0, true));
  return PL_OK;
}

int api_launch_binned(const MatrixF32& M, const int* idx, const long long* offsets, long long nsets,
                      int form, const SetOutputs& out, void* scratch, cudaStream_t st,
                      const cudaStream_t* side, cudaEvent_t fork, const cudaEvent_t* join,
                      const long long* nsets_dev) {
  const bool all = out.eig || out.det;
  size_t qoff[kNumBins];
  binned_qscratch(form, all, qoff);
  LaunchFn fns[kNumBins];
  binned_fns(form, all, fns);
  char* base = (char*)scratch;
  int* hdr = (int*)base;
  char* q = base + align256(sizeof(int) * (48 + (size_t)nsets));
  PL_CU(enqueue_binned(M, idx, offsets, nsets, out, fns, hdr, q, qoff, st, side, fork, join, nsets_dev));
  return PL_OK;
}
void api_note_cuda(cudaError_t e) { g_last_cuda = (int)e; }
int api_device_sms() { return device_sms(); }

// 64-bit content hash of n doubles (their bit patterns): per chunk four
// independent multiply-rotate accumulators over the words, in the style of the
// rounds of Collet's xxHash64 (a published non-cryptographic hash), folded and
// mixed; chunks of 512 KB are spread over up to 16 host threads and their
// hashes combined in chunk order.  At memory speed: a few ms for 128 MB.
static uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static inline uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

static uint64_t hash_chunk(const double* p, size_t n, uint64_t seed) {
  const uint64_t P1 = 0x9E3779B185EBCA87ull, P2 = 0xC2B2AE3D27D4EB4Full;
  uint64_t a0 = seed + P1 + P2, a1 = seed + P2, a2 = seed, a3 = seed - P1;
  const uint64_t* w = reinterpret_cast<const uint64_t*>(p);
  size_t i = 0;
  for (; i + 4 <= n; i += 4) {
    a0 = rotl64(a0 + w[i] * P2, 31) * P1;
    a1 = rotl64(a1 + w[i + 1] * P2, 31) * P1;
    a2 = rotl64(a2 + w[i + 2] * P2, 31) * P1;
    a3 = rotl64(a3 + w[i + 3] * P2, 31) * P1;
  }
  uint64_t h = rotl64(a0, 1) + rotl64(a1, 7) + rotl64(a2, 12) + rotl64(a3, 18);
  for (; i < n; ++i) h = rotl64(h ^ (w[i] * P2), 27) * P1;
  return mix64(h ^ (uint64_t)n);
}

static uint64_t hash_doubles(const double* p, size_t n) {
  const size_t kChunk = size_t(1) << 16;  // 512 KB per chunk
  const size_t nchunks = (n + kChunk - 1) / kChunk;
  std::vector<uint64_t> hs(nchunks ? nchunks : 1, 0);
  unsigned nt = std::thread::hardware_concurrency();
  nt = nt < 1 ? 1 : (nt > 16 ? 16 : nt);
  if (nchunks < 8) nt = 1;  // under 4 MB one thread is as fast as starting more
  if (nt > nchunks) nt = (unsigned)nchunks;
  auto work = [&](unsigned t) {
    for (size_t c = t; c < nchunks; c += nt) {
      const size_t b = c * kChunk, e = b + kChunk < n ? b + kChunk : n;
      hs[c] = hash_chunk(p + b, e - b, c);
    }
  };
  if (nt <= 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& t : th) t.join();
  }
  uint64_t h = mix64(n);
  for (uint64_t x : hs) h = mix64(h ^ x);
  return h;
}

// The drop-in entry points' solve (ParaLanczos.cu:1811-1863 uploads the FP64
// matrix on every call): the FP64 host matrix is uploaded and converted to
// FP32 on the device once, and reused while the caller passes the same
// address, order and contents (PL_DROPIN_CACHE=0 re-uploads every call); the
// index sets go up, all k eigenvalues and the determinants (and per-set
// status) come back.  When the address and order match the cached matrix, the
// solve starts on the cached copy at once and the contents are hashed on the
// host while it runs; a changed hash re-uploads the matrix and solves again
// before anything is copied back.  Synchronous on the legacy default stream,
// like the reference.
int api_solve_f64_host(const double* mat, int n, const int* subIndex, long long nsets, int k, int form,
                       double* eig, double* det, int* err) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!mat || !subIndex || n <= 0 || nsets < 0 || k < 1 || k > n) return PL_EINVAL;
  if (nsets == 0) return PL_OK;
  DevState& d = state();
  cudaStream_t st = 0;
  const size_t nn = (size_t)n * (size_t)n;
  static const bool cache_on = env_flag("PL_DROPIN_CACHE", true);
  auto upload = [&](uint64_t h) -> int {
    d.mc.valid = false;
    int rc = ensure(d.mat64, sizeof(double) * nn);
    if (rc) return rc;
    rc = ensure(d.mat32, sizeof(float) * nn);
    if (rc) return rc;
    PL_CU(cudaMemcpyAsync(d.mat64.p, mat, sizeof(double) * nn, cudaMemcpyHostToDevice, st));
    const long long g = ((long long)nn + 255) / 256;
    k_f64_to_f32<<<(unsigned)(g < 8192 ? g : 8192), 256, 0, st>>>((const double*)d.mat64.p, (float*)d.mat32.p,
                                                                (long long)nn);
    PL_CU(cudaGetLastError());
    d.mc.host = mat;
    d.mc.n = n;
    d.mc.hash = h;
    d.mc.valid = cache_on;
    ++d.mc.misses;
    return PL_OK;
  };
  const bool speculate = cache_on && d.mc.valid && d.mc.host == mat && d.mc.n == n;
  if (!speculate) {
    const int rc = upload(cache_on ? hash_doubles(mat, nn) : 0);
    if (rc) return rc;
  }
  const long long total = nsets * (long long)k;
  const size_t bytes = align256(sizeof(int) * total) + align256(sizeof(double) * total) +
                       align256(sizeof(double) * nsets) + align256(sizeof(int) * nsets) + 1024;
  int rc = ensure(d.upload, bytes);
  if (rc) return rc;
  Carve cv{(char*)d.upload.p, 0};
  int* dI = cv.take<int>(total);
  double* deig = cv.take<double>(total);
  double* ddet = cv.take<double>(nsets);
  int* derr = cv.take<int>(nsets);
  PL_CU(cudaMemcpyAsync(dI, subIndex, sizeof(int) * total, cudaMemcpyHostToDevice, st));
  SetOutputs out{nullptr, nullptr, nullptr, derr, deig, ddet};
  rc = solve_dev((const float*)d.mat32.p, n, n, dI, nullptr, nsets, k, form, out, st);
  if (rc) return rc;
  if (speculate) {
    const uint64_t h = hash_doubles(mat, nn);  // overlaps the solve
    if (h == d.mc.hash) {
      ++d.mc.hits;
    } else {
      rc = upload(h);
      if (rc) return rc;
      rc = solve_dev((const float*)d.mat32.p, n, n, dI, nullptr, nsets, k, form, out, st);
      if (rc) return rc;
    }
  }
  if (eig) PL_CU(cudaMemcpyAsync(eig, deig, sizeof(double) * total, cudaMemcpyDeviceToHost, st));
  if (det) PL_CU(cudaMemcpyAsync(det, ddet, sizeof(double) * nsets, cudaMemcpyDeviceToHost, st));
  if (err) PL_CU(cudaMemcpyAsync(err, derr, sizeof(int) * nsets, cudaMemcpyDeviceToHost, st));
  PL_CU(cudaStreamSynchronize(st));
  return PL_OK;
}

void api_dropin_cache_stats(long long* hits, long long* misses) {
  std::lock_guard<std::mutex> lk(g_mu);
  const DevState& d = state();
  if (hits) *hits = d.mc.hits;
  if (misses) *misses = d.mc.misses;
}
}  // namespace pl

// =============================================================================
// Allocation-free entry point (pl_solve_noalloc)
// =============================================================================
// Some callers cannot call cudaMalloc: a host that owns the device memory
// budget (an embedding runtime or a serving process that pre-partitions HBM),
// code running while a CUDA graph is being captured, or a plugin whose
// contract forbids allocation after start-up.  For them the batched k <= 64
// kernels can run with their deferred-bisection queues in this file-scope
// array instead of a cudaMalloc'd buffer.  32 MiB covers the full persistent
// grid of every k <= 64 kernel; every GPU that loads the library holds the
// array until the process exits.  All calls share it and it keeps the last
// call's contents (nothing in it has to start at zero: a queue slot is written
// before it is read), so calls whose kernels overlap on the GPU race.
constexpr size_t kNoAllocBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {
void* g_noalloc_ptr[64] = {};

// Once per device, with that device current: the array's device address (the
// symbol itself is only a host-side stand-in).
int noalloc_setup(void** out) {
  int dev = 0;
  PL_CU(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return PL_ENOTSUP;
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    PL_CU(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return PL_OK;
}
}  // namespace

// =============================================================================
// C ABI
// =============================================================================
extern "C" {

int pl_version(void) { return 100; }

const char* pl_status_string(int s) {
  switch (s) {
    case PL_OK: return "ok";
    case PL_EINVAL: return "invalid argument";
    case PL_ECUDA: return "CUDA error";
    case PL_ENOMEM: return "out of memory";
    case PL_ENOTSUP: return "not supported";
    case PL_ETIMEDOUT: return "timed out";
    case PL_EBUSY: return "busy";
    default: return "unknown status";
  }
}

int pl_last_cuda_error(void) { return g_last_cuda; }

int pl_solve(const float* A, int n, long long lda, const int* idx, const long long* offsets,
             long long nsets, int k, int form, double* lmin, double* lmax, double* delta, int* err,
             double* eig, double* det, void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  SetOutputs out{lmin, lmax, delta, err, eig, det};
  return solve_dev(A, n, lda, idx, offsets, nsets, k, form, out, (cudaStream_t)stream);
}

int pl_solve_noalloc(const float* A, int n, long long lda, const int* idx, long long nsets, int k,
                     double* lmin, double* lmax, double* delta, int* err, void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  int rc = validate_common(A, n, lda, idx, nsets, k, nullptr, PL_FORM_BATCHED);
  if (rc || nsets == 0) return rc;
  const int b = bin_of_k(k);
  if (b < 0 || kBinK[b] > 64) return PL_ENOTSUP;  // only the k <= 64 kernels fit the array
  const Variant& v = chosen(b);
  if (v.scratch[0]() > kNoAllocBytes) return PL_ENOTSUP;
  void* scratch = nullptr;
  rc = noalloc_setup(&scratch);
  if (rc) return rc;
  MatrixF32 M{A, lda, n};
  SetSource src{idx, nullptr, k, nullptr, nullptr, nullptr, nsets};
  SetOutputs out{lmin, lmax, delta, err, nullptr, nullptr};
  PL_CU(v.fn[0](M, src, out, nsets, scratch, (cudaStream_t)stream, false));
  return PL_OK;
}

int pl_solve_host(const float* A, int n, long long lda, const int* idx, const long long* offsets,
                  long long nsets, int k, int form, double* lmin, double* lmax, double* delta,
                  int* err, double* eig, double* det) {
  std::lock_guard<std::mutex> lk(g_mu);
  int rc = validate_common(A, n, lda, idx, nsets, k, offsets, form);
  if (rc || nsets == 0) return rc;
  long long total = offsets ? offsets[nsets] : nsets * (long long)k;
  if (offsets && offsets[0] != 0) return PL_EINVAL;
  const size_t bytes = align256(sizeof(float) * (size_t)n * lda) + align256(sizeof(int) * total) +
                       align256(sizeof(long long) * (nsets + 1)) + 4 * align256(sizeof(double) * nsets) +
                       align256(sizeof(int) * nsets) + align256(sizeof(double) * total) + 4096;
  DevState& d = state();
  rc = ensure(d.upload, bytes);
  if (rc) return rc;
  Carve cv{(char*)d.upload.p, 0};
  float* dA = cv.take<float>((size_t)n * lda);
  int* dI = cv.take<int>(total);
  long long* dO = offsets ? cv.take<long long>(nsets + 1) : nullptr;
  double* dmin = lmin ? cv.take<double>(nsets) : nullptr;
  double* dmax = lmax ? cv.take<double>(nsets) : nullptr;
  double* ddel = delta ? cv.take<double>(nsets) : nullptr;
  double* ddet = det ? cv.take<double>(nsets) : nullptr;
  int* derr = err ? cv.take<int>(nsets) : nullptr;
  double* deig = eig ? cv.take<double>(total) : nullptr;
  cudaStream_t st = 0;
  PL_CU(cudaMemcpyAsync(dA, A, sizeof(float) * (size_t)n * lda, cudaMemcpyHostToDevice, st));
  // Uniform k whose kernel reads each set's indices a whole set ahead (the
  // tuned k <= 64 shape): when the caller's index array is pinned host memory
  // mapped into the device's address space, the kernel reads it over the host
  // link while it computes, instead of waiting for a copy of the whole array
  // before the launch.  Anything else is copied first.
  const int* idx_src = dI;
  if (!offsets && form == PL_FORM_BATCHED && !eig && !det) {
    const int b = bin_of_k(k);
    cudaPointerAttributes pa{};
    if (b >= 0 && chosen(b).indices_ahead && chosen(b).fn[0]) {
      if (cudaPointerGetAttributes(&pa, idx) == cudaSuccess && pa.type == cudaMemoryTypeHost && pa.devicePointer)
        idx_src = (const int*)pa.devicePointer;
      else
        cudaGetLastError();  // pageable memory is not an error
    }
  }
  if (idx_src == dI) PL_CU(cudaMemcpyAsync(dI, idx, sizeof(int) * total, cudaMemcpyHostToDevice, st));
  if (dO) PL_CU(cudaMemcpyAsync(dO, offsets, sizeof(long long) * (nsets + 1), cudaMemcpyHostToDevice, st));
  SetOutputs out{dmin, dmax, ddel, derr, deig, ddet};
  rc = solve_dev(dA, n, lda, idx_src, dO, nsets, k, form, out, st);
  if (rc) return rc;
  if (lmin) PL_CU(cudaMemcpyAsync(lmin, dmin, sizeof(double) * nsets, cudaMemcpyDeviceToHost, st));
  if (lmax) PL_CU(cudaMemcpyAsync(lmax, dmax, sizeof(double) * nsets, cudaMemcpyDeviceToHost, st));
  if (delta) PL_CU(cudaMemcpyAsync(delta, ddel, sizeof(double) * nsets, cudaMemcpyDeviceToHost, st));
  if (det) PL_CU(cudaMemcpyAsync(det, ddet, sizeof(double) * nsets, cudaMemcpyDeviceToHost, st));
  if (err) PL_CU(cudaMemcpyAsync(err, derr, sizeof(int) * nsets, cudaMemcpyDeviceToHost, st));
  if (eig) PL_CU(cudaMemcpyAsync(eig, deig, sizeof(double) * total, cudaMemcpyDeviceToHost, st));
  PL_CU(cudaStreamSynchronize(st));
  return PL_OK;
}

int pl_gather_blocks(const float* A, int n, long long lda, const int* idx, long long nsets, int k,
                     float* blocks, int* err, void* stream) {
  if (nsets < 0 || n <= 0 || lda < n || k < 1 || k > PL_KMAX || k > n) return PL_EINVAL;
  if (nsets == 0) return PL_OK;
  if (!A || !idx || !blocks) return PL_EINVAL;
  const long long g = (long long)device_sms() * 8;
  k_gather_blocks<<<(unsigned)(nsets < g ? nsets : g), 256, 0, (cudaStream_t)stream>>>(A, n, lda, idx, nsets, k,
                                                                                      blocks, err);
  PL_CU(cudaGetLastError());
  return PL_OK;
}

int pl_gen_sets(unsigned long long seed, long long first, long long nsets, int n, int k, int* idx,
                void* stream) {
  if (nsets < 0 || k < 1 || k > n || (nsets > 0 && !idx)) return PL_EINVAL;
  if (nsets == 0) return PL_OK;
  const long long g = (nsets + 255) / 256;
  k_gen_sets<<<(unsigned)(g < 65535 ? g : 65535), 256, 0, (cudaStream_t)stream>>>(seed, first, nsets,
                                                                                   n, k, idx);
  PL_CU(cudaGetLastError());
  return PL_OK;
}

long long pl_gen_stream_host(unsigned long long seed, long long first, long long nsets, int n,
                             int kdist, int kmin, int kmax, long long* offsets, int* idx) {
  long long off = 0;
  for (long long s = 0; s < nsets; ++s) {
    const int k = gen_k(seed, (uint64_t)(first + s), kdist, kmin, kmax);
    if (offsets) offsets[s] = off;
    if (idx) gen_set(seed, (uint64_t)(first + s), n, k, idx + off);
    off += k;
  }
  if (offsets) offsets[nsets] = off;
  return off;
}

int pl_convert_f64_f32(const double* in, float* out, long long count, void* stream) {
  if (count < 0 || (count > 0 && (!in || !out))) return PL_EINVAL;
  if (count == 0) return PL_OK;
  const long long g = (count + 255) / 256;
  k_f64_to_f32<<<(unsigned)(g < 8192 ? g : 8192), 256, 0, (cudaStream_t)stream>>>(in, out, count);
  PL_CU(cudaGetLastError());
  return PL_OK;
}

void pl_dropin_cache_stats(long long* hits, long long* misses) { api_dropin_cache_stats(hits, misses); }

int pl_tune_set(int bin, int variant) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (bin < 0 || bin >= kNumBins) return PL_EINVAL;
  if (variant >= (int)variants(bin).size()) return PL_EINVAL;
  g_variant[bin] = variant < 0 ? kDefaultVariant[bin] : variant;
  return PL_OK;
}

int pl_tune_get(int bin) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (bin < 0 || bin >= kNumBins) return -1;
  return g_variant[bin];
}

int pl_tune_describe(int bin, int variant, char* buf, int buflen) {
  if (bin < 0 || bin >= kNumBins) return 0;
  const auto& v = variants(bin);
  if (buf && buflen > 0) {
    const char* s = (variant >= 0 && variant < (int)v.size()) ? v[variant].desc : "";
    snprintf(buf, (size_t)buflen, "%s", s);
  }
  return (int)v.size();
}

int pl_num_bins(void) { return kNumBins; }

int pl_bin_kmax(int bin) { return (bin >= 0 && bin < kNumBins) ? kBinK[bin] : 0; }

int pl_fp32_peak(double* tflops, void* stream) {
  if (!tflops) return PL_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  float* dummy = nullptr;
  PL_CU(cudaMalloc(&dummy, 256 * sizeof(float)));
  cudaEvent_t e0, e1;
  PL_CU(cudaEventCreate(&e0));
  PL_CU(cudaEventCreate(&e1));
  const int grid = device_sms() * 8, iters = 2048;
  k_fma_peak<<<grid, 256, 0, st>>>(dummy, iters, 0.999f);  // warm-up
  cudaEventRecord(e0, st);
  k_fma_peak<<<grid, 256, 0, st>>>(dummy, iters, 0.999f);
  cudaEventRecord(e1, st);
  PL_CU(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(dummy);
  const double flops = 2.0 * 8 * 16 * (double)iters * grid * 256;
  *tflops = flops / (ms * 1e-3) / 1e12;
  PL_CU(cudaGetLastError());
  return PL_OK;
}

int pl_gather_peak(double* gelems, void* stream) {
  if (!gelems) return PL_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  float* buf = nullptr;
  PL_CU(cudaMalloc(&buf, sizeof(float) * ((size_t)1 << 24) + 256));
  cudaError_t e = cudaMemsetAsync(buf, 0, sizeof(float) * ((size_t)1 << 24) + 256, st);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  const int grid = device_sms() * 4, iters = 200;
  float ms = 0.f;
  if (e == cudaSuccess) {
    k_gather_peak<<<grid, 256, 0, st>>>(buf, 20, buf + ((size_t)1 << 24));  // warm-up: A into L2
    cudaEventRecord(e0, st);
    k_gather_peak<<<grid, 256, 0, st>>>(buf, iters, buf + ((size_t)1 << 24));
    cudaEventRecord(e1, st);
    e = cudaEventSynchronize(e1);
  }
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(buf);
  PL_CU(e);
  *gelems = 16.0 * iters * (double)grid * 256 / (ms * 1e-3) / 1e9;
  return PL_OK;
}

int pl_release(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  cudaDeviceSynchronize();
  DevState& d = state();
  for (auto& kv : d.graphs) cudaGraphExecDestroy(kv.second.exec);
  d.graphs.clear();
  for (DevScratch* s : {&d.large, &d.bins, &d.upload, &d.mat64, &d.mat32}) {
    if (s->p) cudaFree(s->p);
    s->p = nullptr;
    s->bytes = 0;
  }
  d.mc.valid = false;
  gram_release();
  return PL_OK;
}

}  // extern "C"
