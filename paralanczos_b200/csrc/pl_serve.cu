// pl_serve.cu -- serving: continuous batching in a device-resident request loop.
//
// The reference has no serving layer: each calculate_subeigs* call
// (ParaLanczos.cu:1725-1863) uploads one matrix and one batch of sets,
// launches, copies back and resets the device.  Here a server keeps several
// matrices resident and solves requests -- (matrix, k, a batch of index sets)
// -- as they arrive, with the batching done on the GPU:
//
//   * submit() copies the request's indices into a pinned (device-mapped)
//     host pool and queues it (PL_EBUSY when the pool is full: back-pressure);
//   * the host admits queued requests in arrival order while their indices
//     fit the device arena, uploads them, and then publishes one descriptor
//     per request into a descriptor ring in mapped host memory;
//   * request loops run on the device, up to four: each is one CUDA graph whose
//     body sits under a conditional WHILE node -- a planning kernel, an
//     expansion kernel, the binned launch of the batched form (device counting
//     sort by k, one persistent kernel per k bin), and a completion kernel --
//     and repeats without the host.  The loops share one table of active
//     requests in device memory: each pass a loop's planning kernel absorbs new
//     descriptors from the ring (claiming each with a compare-and-swap), scans
//     the table with a whole CTA, and forms its next "wave" of about
//     PL_SERVE_WAVE_MS (default 10) ms of estimated GPU work -- the oldest
//     unfinished request gets up to PL_SERVE_OLDEST_SHARE (default 0.9) of it,
//     then the requests with the least work left fill the rest -- claiming the
//     sets with atomic adds, so two loops never take the same set and no kernel
//     waits on another.  With several loops, several waves are in flight and
//     their kernels overlap (one wave's tail is filled by the next), in one
//     global oldest-first order: large requests are split over waves and are
//     not stretched by sharing, small ones that arrive behind them go out in
//     the next wave.  The expansion kernel lays a wave's sets out as one CSR
//     batch (indices copied from the arena, per-set matrix ids); the completion
//     kernel writes each set's results straight into its request's mapped host
//     buffers and, with the last set of a request, its completion flag;
//   * when a loop finds nothing to do, its planning kernel polls the ring
//     (bounded by %globaltimer, PL_SERVE_IDLE_MS, default 20 ms) and then ends
//     the loop (the graph finishes, status "idle"); the host launches it again
//     when the next descriptor is published.  Every device wait is bounded;
//   * all device memory of the server -- arena, wave staging, kernel scratch,
//     tables -- is allocated at creation inside budget_bytes.
// A set's result does not depend on what else is in its wave: each set is
// solved by its bin's kernel on its own data with a fixed reduction order.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/paralanczos.h"
#include "pl_common.cuh"
#include "pl_internal.h"
#include "pl_serve_plan.cuh"
#include "pl_sync.cuh"

namespace pl {
namespace serve {

constexpr int kMaxMatrices = 64;
constexpr int kMaxBinsS = 16;
constexpr int kRing = 4096;  // descriptor ring entries

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

// First-fit allocator over [0, size) with coalescing free blocks.
struct Arena {
  size_t size = 0;
  std::map<size_t, size_t> free_;  // offset -> length
  size_t used = 0, peak = 0;
  void init(size_t n) {
    size = n;
    free_.clear();
    if (n) free_[0] = n;
    used = peak = 0;
  }
  bool alloc(size_t n, size_t* off) {
    n = a256(n ? n : 1);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= n) {
        *off = it->first;
        const size_t rest = it->second - n;
        const size_t noff = it->first + n;
        free_.erase(it);
        if (rest) free_[noff] = rest;
        used += n;
        peak = std::max(peak, used);
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t n) {
    n = a256(n ? n : 1);
    used -= n;
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
};

struct LoopArgs {
  Ctl* ctl;              // mapped
  const RingDesc* ring;  // mapped
  Shared* sh;            // device, shared by the loops
  Plan* plan;            // device, this loop's
  const int* arena;
  int* widx;
  long long* woff;
  int* wmat;
  int* wslot;
  long long* wpos;
  double* wres;  // lmin, lmax, delta: kWaveSets each
  int* werr;
  cudaGraphConditionalHandle cond;
  unsigned long long idle_ns;
  double wave_us, oldest_share;
  int loop;
};

__device__ __forceinline__ long long ld_acquire_sys(const long long* p) {
  long long v;
  asm volatile("ld.acquire.sys.global.s64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_sys(long long* p, long long v) {
  asm volatile("st.release.sys.global.s64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void st_release_gpu(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// New descriptors into the shared table (one thread).  Each ring entry is
// claimed by exactly one planner (compare-and-swap on the shared cursor); the
// request becomes visible to the scans by a release store of `live` after its
// fields.
__device__ void absorb(const LoopArgs& a) {
  const long long tail = ld_acquire_sys(&a.ctl->tail);
  for (int it = 0; it < kRing; ++it) {
    const unsigned long long h = *(volatile unsigned long long*)&a.sh->head;
    if ((long long)h >= tail) break;
    if (atomicCAS(&a.sh->head, h, h + 1) != h) continue;
    const RingDesc d = a.ring[h % kRing];
    DevReq& r = a.sh->tab[d.slot];
    r.id = d.id;
    r.nsets = d.nsets;
    r.next = 0;
    r.done = 0;
    r.arena_off = d.arena_off;
    r.lmin = d.lmin;
    r.lmax = d.lmax;
    r.delta = d.delta;
    r.err = d.err;
    r.mat = d.mat;
    r.k = d.k;
    st_release_gpu(&r.live, 1);
    *(volatile long long*)&a.ctl->head = (long long)h + 1;
  }
}

// Planning (one CTA of 256 threads): absorb, scan the table for requests with
// sets left, wait for work at most idle_ns, then form this loop's next wave
// (thread 0) or end the loop.
__global__ void __launch_bounds__(256) k_loop_plan(LoopArgs a) {
  __shared__ Cand cand[kSlots];
  __shared__ int nc, decision;
  const unsigned long long t0 = globaltimer();
  for (;;) {
    if (threadIdx.x == 0) {
      absorb(a);
      nc = 0;
    }
    __syncthreads();
    for (int s = threadIdx.x; s < kSlots; s += blockDim.x) {
      const DevReq& r = a.sh->tab[s];
      if (ld_acquire_gpu(&r.live)) {
        const long long nx = *(volatile const long long*)&r.next;
        if (nx < r.nsets) {
          const int i = atomicAdd(&nc, 1);
          cand[i] = Cand{r.id, r.nsets - nx, s, r.k};
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int stop = *(volatile int*)&a.ctl->stop;
      decision = (nc > 0 && !stop) ? 1 : ((stop || globaltimer() - t0 > a.idle_ns) ? 2 : 0);
      if (decision == 0) __nanosleep(2000);
    }
    __syncthreads();
    if (decision == 1) break;
    if (decision == 2) {
      if (threadIdx.x == 0) {
        a.plan->nsets = 0;
        a.plan->npieces = 0;
        *(volatile int*)&a.ctl->status[a.loop] = *(volatile int*)&a.ctl->stop ? 3 : 2;
        cudaGraphSetConditional(a.cond, 0);
      }
      return;
    }
  }
  if (threadIdx.x != 0) return;
  auto claim = [&](int slot, long long want, long long* first) -> long long {
    DevReq& r = a.sh->tab[slot];
    const long long old = (long long)atomicAdd(reinterpret_cast<unsigned long long*>(&r.next),
                                               (unsigned long long)want);
    if (old >= r.nsets) return 0;
    *first = old;
    return want < r.nsets - old ? want : r.nsets - old;
  };
  long long ns = 0;
  a.plan->npieces = form_wave(cand, nc, a.wave_us, a.oldest_share, a.plan->pieces, &ns, claim);
  a.plan->nsets = ns;
  *(volatile long long*)&a.ctl->waves[a.loop] = *(volatile long long*)&a.ctl->waves[a.loop] + 1;
  cudaGraphSetConditional(a.cond, 1);  // an empty wave (claims lost to other loops) plans again
}

// The wave as one CSR batch: a warp per set copies its indices from the arena.
__global__ void __launch_bounds__(256) k_loop_expand(LoopArgs a) {
  const Plan& P = *a.plan;
  const long long ns = P.nsets;
  const int lane = threadIdx.x & 31;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long s = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < ns; s += nw) {
    int lo = 0, hi = P.npieces - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (P.pieces[mid].set0 <= s) lo = mid; else hi = mid - 1;
    }
    const Piece pc = P.pieces[lo];
    const long long j = s - pc.set0, pos = pc.first + j, off = pc.idx0 + j * pc.k;
    const DevReq& r = a.sh->tab[pc.slot];
    const int* __restrict__ src = a.arena + r.arena_off + pos * pc.k;
    for (int i = lane; i < pc.k; i += 32) a.widx[off + i] = src[i];
    if (lane == 0) {
      a.woff[s] = off;
      a.wmat[s] = r.mat;
      a.wslot[s] = pc.slot;
      a.wpos[s] = pos;
      if (s == ns - 1) a.woff[ns] = off + pc.k;
    }
  }
}

// Results into the requests' mapped host buffers; the last set of a request
// retires it (live = 0) and then publishes its completion flag, after every
// result of it is visible to the host.
__global__ void __launch_bounds__(256) k_loop_finish(LoopArgs a) {
  const long long ns = a.plan->nsets;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < ns;
       s += (long long)gridDim.x * blockDim.x) {
    const int slot = a.wslot[s];
    const long long pos = a.wpos[s];
    DevReq& r = a.sh->tab[slot];
    r.lmin[pos] = a.wres[s];
    r.lmax[pos] = a.wres[kWaveSets + s];
    r.delta[pos] = a.wres[2 * kWaveSets + s];
    r.err[pos] = a.werr[s];
    __threadfence_system();
    const unsigned long long prev = atomicAdd(reinterpret_cast<unsigned long long*>(&r.done), 1ull);
    if ((long long)prev + 1 == r.nsets) {
      *(volatile int*)&r.live = 0;
      __threadfence_system();
      st_release_sys(&a.ctl->done_id[slot], r.id);
    }
  }
}

// ---- host side ------------------------------------------------------------------
enum ReqState { PENDING = 0, UPLOADING = 1, PUBLISHED = 2, DONE = 3, FAILED = 4 };

struct Request {
  long long id = 0;
  int mat = 0, k = 0;
  long long nsets = 0;
  size_t host_off = 0, host_len = 0;  // pinned pool block: idx, then results
  int* h_idx = nullptr;
  double* h_res = nullptr;  // lmin[nsets], lmax[nsets], delta[nsets]
  int* h_err = nullptr;
  double t_submit = 0, t_done = 0;
  int state = PENDING;
  int status = PL_OK;
  size_t dev_off = 0, dev_len = 0;  // arena block holding the indices on the device
  int slot = -1;
};

size_t req_dev_bytes(long long nsets, int k) { return a256(sizeof(int) * (size_t)nsets * k); }
size_t req_host_bytes(long long nsets, int k) {
  return a256(sizeof(int) * (size_t)nsets * k) + a256(3 * sizeof(double) * (size_t)nsets) +
         a256(sizeof(int) * (size_t)nsets);
}

struct Loop {
  Plan* plan = nullptr;
  char* dmem = nullptr;  // one device allocation: plan, wave staging, scratch
  LoopArgs args{};
  void* scratch = nullptr;
  cudaStream_t st = nullptr, cap = nullptr;
  cudaStream_t side[kMaxBinsS] = {};
  cudaEvent_t fork = nullptr, join[kMaxBinsS] = {};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool running = false;
  long long launches = 0, idle_exits = 0;
};

struct Server {
  int dev = 0, nbins = 0, nloops = 1;
  Arena arena;  // device budget left for request indices
  char* d_arena = nullptr;
  Arena pool;   // pinned host staging (device-mapped)
  char* h_pool = nullptr;
  char* d_pool = nullptr;  // the pool's device address
  MatrixRef* d_mats = nullptr;
  std::vector<MatrixRef> mats;
  Shared* sh = nullptr;    // device: the shared request table
  Ctl* ctl = nullptr;      // mapped
  RingDesc* ring = nullptr;  // mapped
  Ctl* ctl_d = nullptr;
  RingDesc* ring_d = nullptr;
  long long published = 0;
  std::vector<int> free_slots;
  std::vector<Request*> live;  // published, not complete
  Loop loops[kMaxLoops];
  size_t fixed_bytes = 0, budget = 0;
  cudaStream_t up = nullptr;  // index uploads at admission
  cudaEvent_t up_ev = nullptr;
  std::vector<Request*> uploading;  // uploaded by up_ev, not yet published
  double wave_us = 10000.0, oldest_share = 0.9, idle_ms = 20.0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> pending;  // submitted, not admitted (arrival order)
  std::unordered_map<long long, Request*> reqs;
  std::thread th;
  std::atomic<bool> stop{false};
  long long next_id = 1;
  std::vector<double> lat;
  long long sets_done = 0;
  int running_max = 0;
  double t_first = 0, t_last = 0;
};

int cuda_fail(cudaError_t e) {
  api_note_cuda(e);
  return e == cudaErrorMemoryAllocation ? PL_ENOMEM : PL_ECUDA;
}

// Device bytes of one loop (its wave, wave staging, binned-launch scratch).
struct LoopLayout {
  size_t plan, widx, woff, wmat, wslot, wpos, wres, werr, scratch, total;
};
LoopLayout loop_layout() {
  LoopLayout L;
  size_t o = 0;
  auto take = [&](size_t n) {
    const size_t at = o;
    o += a256(n);
    return at;
  };
  L.plan = take(sizeof(Plan));
  L.widx = take(sizeof(int) * (size_t)kWaveIdx);
  L.woff = take(sizeof(long long) * (size_t)(kWaveSets + 1));
  L.wmat = take(sizeof(int) * (size_t)kWaveSets);
  L.wslot = take(sizeof(int) * (size_t)kWaveSets);
  L.wpos = take(sizeof(long long) * (size_t)kWaveSets);
  L.wres = take(3 * sizeof(double) * (size_t)kWaveSets);
  L.werr = take(sizeof(int) * (size_t)kWaveSets);
  L.scratch = take(api_binned_scratch(kWaveSets, PL_FORM_BATCHED, false));
  L.total = o;
  return L;
}

// A loop's graph: WHILE(cond) { plan; expand; binned solve; finish }.
int build_loop(Server& S, Loop& L, int li) {
  const LoopLayout lay = loop_layout();
  cudaError_t e;
  if ((e = cudaMalloc(&L.dmem, lay.total)) != cudaSuccess) return cuda_fail(e);
  if ((e = cudaMemset(L.dmem + lay.plan, 0, sizeof(Plan))) != cudaSuccess) return cuda_fail(e);
  L.plan = (Plan*)(L.dmem + lay.plan);
  L.scratch = L.dmem + lay.scratch;
  LoopArgs& a = L.args;
  a.ctl = S.ctl_d;
  a.ring = S.ring_d;
  a.sh = S.sh;
  a.plan = L.plan;
  a.arena = (const int*)S.d_arena;
  a.widx = (int*)(L.dmem + lay.widx);
  a.woff = (long long*)(L.dmem + lay.woff);
  a.wmat = (int*)(L.dmem + lay.wmat);
  a.wslot = (int*)(L.dmem + lay.wslot);
  a.wpos = (long long*)(L.dmem + lay.wpos);
  a.wres = (double*)(L.dmem + lay.wres);
  a.werr = (int*)(L.dmem + lay.werr);
  a.idle_ns = (unsigned long long)(S.idle_ms * 1e6);
  a.wave_us = S.wave_us;
  a.oldest_share = S.oldest_share;
  a.loop = li;
  if ((e = cudaStreamCreateWithFlags(&L.st, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&L.cap, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&L.fork, cudaEventDisableTiming)) != cudaSuccess)
    return cuda_fail(e);
  for (int b = 0; b < S.nbins; ++b)
    if ((e = cudaStreamCreateWithFlags(&L.side[b], cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&L.join[b], cudaEventDisableTiming)) != cudaSuccess)
      return cuda_fail(e);

  if ((e = cudaGraphCreate(&L.graph, 0)) != cudaSuccess) return cuda_fail(e);
  if ((e = cudaGraphConditionalHandleCreate(&a.cond, L.graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess)
    return cuda_fail(e);
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = a.cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if ((e = cudaGraphAddNode(&node, L.graph, nullptr, 0, &cp)) != cudaSuccess) return cuda_fail(e);
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  int rc;
  {
    std::lock_guard<std::mutex> lk(api_mutex());
    rc = api_prepare_binned(PL_FORM_BATCHED, false);
  }
  if (rc) return rc;
  const int sms = api_device_sms();
  if ((e = cudaStreamBeginCaptureToGraph(L.cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
      cudaSuccess)
    return cuda_fail(e);
  k_loop_plan<<<1, 256, 0, L.cap>>>(a);
  k_loop_expand<<<sms * 4, 256, 0, L.cap>>>(a);
  MatrixF32 M{nullptr, 0, 0};
  M.mats = S.d_mats;
  M.mat_id = a.wmat;
  SetOutputs out{a.wres, a.wres + kWaveSets, a.wres + 2 * kWaveSets, a.werr, nullptr, nullptr};
  {
    std::lock_guard<std::mutex> lk(api_mutex());
    rc = api_launch_binned(M, a.widx, a.woff, kWaveSets, PL_FORM_BATCHED, out, L.scratch, L.cap, L.side, L.fork,
                           L.join, &L.plan->nsets);
  }
  k_loop_finish<<<sms * 4, 256, 0, L.cap>>>(a);
  cudaGraph_t captured = nullptr;
  e = cudaStreamEndCapture(L.cap, &captured);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e);
  if ((e = cudaGraphInstantiate(&L.exec, L.graph, 0)) != cudaSuccess) return cuda_fail(e);
  return PL_OK;
}

void fail_live(Server& S, int status) {
  const double t = now_s();
  for (Request* r : S.live) {
    r->state = FAILED;
    r->status = status;
    r->t_done = t;
    S.arena.release(r->dev_off, r->dev_len);
    S.free_slots.push_back(r->slot);
  }
  S.live.clear();
}

void scheduler(Server* sp) {
  Server& S = *sp;
  cudaSetDevice(S.dev);
  std::unique_lock<std::mutex> lk(S.mu);
  while (!S.stop.load()) {
    bool progressed = false;
    // ---- completions: flags written by the device loops
    const double t = now_s();
    for (size_t i = 0; i < S.live.size();) {
      Request* r = S.live[i];
      if (*(volatile long long*)&S.ctl->done_id[r->slot] == r->id) {
        r->state = DONE;
        r->t_done = t;
        S.lat.push_back(t - r->t_submit);
        S.t_last = t;
        S.sets_done += r->nsets;
        S.arena.release(r->dev_off, r->dev_len);
        S.free_slots.push_back(r->slot);
        S.live[i] = S.live.back();
        S.live.pop_back();
        progressed = true;
      } else {
        ++i;
      }
    }
    if (progressed) S.cv_done.notify_all();
    // ---- publication of the uploaded batch (in arrival order)
    if (!S.uploading.empty() && cudaEventQuery(S.up_ev) == cudaSuccess) {
      for (Request* r : S.uploading) {
        RingDesc& d = S.ring[S.published % kRing];
        const size_t nres = (size_t)r->nsets;
        double* res = (double*)(S.d_pool + ((char*)r->h_res - S.h_pool));
        int* err = (int*)(S.d_pool + ((char*)r->h_err - S.h_pool));
        d = RingDesc{r->id, r->nsets, (long long)(r->dev_off / sizeof(int)), res, res + nres, res + 2 * nres,
                     err, r->slot, r->mat, r->k, 0};
        std::atomic_thread_fence(std::memory_order_release);
        ++S.published;
        *(volatile long long*)&S.ctl->tail = S.published;
        r->state = PUBLISHED;
        S.live.push_back(r);
      }
      S.uploading.clear();
      progressed = true;
    }
    // ---- admission: arrival order, while the indices fit the arena, a slot
    //      is free and the ring has room (a margin for entries being copied)
    if (S.uploading.empty()) {
      while (!S.pending.empty()) {
        Request* r = S.pending.front();
        if (S.free_slots.empty()) break;
        if (S.published + (long long)S.uploading.size() - *(volatile long long*)&S.ctl->head >= kRing - 64) break;
        size_t off = 0;
        const size_t b = req_dev_bytes(r->nsets, r->k);
        if (!S.arena.alloc(b, &off)) break;
        r->dev_off = off;
        r->dev_len = b;
        r->slot = S.free_slots.back();
        S.free_slots.pop_back();
        r->state = UPLOADING;
        cudaError_t e = cudaMemcpyAsync(S.d_arena + off, r->h_idx, sizeof(int) * (size_t)r->nsets * r->k,
                                        cudaMemcpyHostToDevice, S.up);
        if (e != cudaSuccess) api_note_cuda(e);
        S.pending.pop_front();
        S.uploading.push_back(r);
      }
      if (!S.uploading.empty()) {
        cudaEventRecord(S.up_ev, S.up);
        if (S.t_first == 0) S.t_first = now_s();
        progressed = true;
      }
    }
    // ---- the device loops: notice ended ones, (re)launch while work is live
    int running = 0;
    for (int li = 0; li < S.nloops; ++li) {
      Loop& L = S.loops[li];
      if (L.running) {
        const cudaError_t q = cudaStreamQuery(L.st);
        if (q == cudaSuccess) {
          L.running = false;
          if (*(volatile int*)&S.ctl->status[li] == 2) ++L.idle_exits;
        } else if (q != cudaErrorNotReady) {
          api_note_cuda(q);
          L.running = false;
          fail_live(S, PL_ECUDA);
          S.cv_done.notify_all();
        }
      }
      if (!L.running && !S.live.empty()) {
        *(volatile int*)&S.ctl->status[li] = 1;
        std::atomic_thread_fence(std::memory_order_release);
        const cudaError_t e = cudaGraphLaunch(L.exec, L.st);
        if (e != cudaSuccess) {
          api_note_cuda(e);
          fail_live(S, PL_ECUDA);
          S.cv_done.notify_all();
        } else {
          L.running = true;
          ++L.launches;
          progressed = true;
        }
      }
      running += L.running ? 1 : 0;
    }
    S.running_max = std::max(S.running_max, running);
    if (!progressed) {
      if (!S.uploading.empty() || !S.live.empty()) {
        lk.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(20));
        lk.lock();
      } else {
        S.cv_work.wait_for(lk, std::chrono::milliseconds(2));
      }
    }
  }
}

int destroy(Server* S) {
  if (!S) return PL_EINVAL;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop.store(true);
  }
  S->cv_work.notify_all();
  if (S->th.joinable()) S->th.join();
  cudaSetDevice(S->dev);
  if (S->ctl) *(volatile int*)&S->ctl->stop = 1;  // a running loop leaves at its next poll
  for (int li = 0; li < kMaxLoops; ++li) {
    Loop& L = S->loops[li];
    if (L.st) cudaStreamSynchronize(L.st);
    if (L.exec) cudaGraphExecDestroy(L.exec);
    if (L.graph) cudaGraphDestroy(L.graph);
    for (int b = 0; b < kMaxBinsS; ++b) {
      if (L.side[b]) cudaStreamDestroy(L.side[b]);
      if (L.join[b]) cudaEventDestroy(L.join[b]);
    }
    if (L.st) cudaStreamDestroy(L.st);
    if (L.cap) cudaStreamDestroy(L.cap);
    if (L.fork) cudaEventDestroy(L.fork);
    if (L.dmem) cudaFree(L.dmem);
  }
  if (S->up) cudaStreamSynchronize(S->up);
  if (S->up) cudaStreamDestroy(S->up);
  if (S->up_ev) cudaEventDestroy(S->up_ev);
  for (auto& kv : S->reqs) delete kv.second;
  if (S->d_arena) cudaFree(S->d_arena);
  if (S->d_mats) cudaFree(S->d_mats);
  if (S->sh) cudaFree(S->sh);
  if (S->ctl) cudaFreeHost(S->ctl);
  if (S->ring) cudaFreeHost(S->ring);
  if (S->h_pool) cudaFreeHost(S->h_pool);
  delete S;
  return PL_OK;
}

}  // namespace serve
}  // namespace pl

using namespace pl;
using namespace pl::serve;

extern "C" {

int pl_serve_create(long long budget_bytes, long long host_pool_bytes, int max_waves, void** server) {
  if (!server || budget_bytes < 4096 || host_pool_bytes < 4096 || max_waves < 1 || max_waves > 8)
    return PL_EINVAL;
  *server = nullptr;
  const int nloops = std::min(max_waves, kMaxLoops);
  const size_t fixed =
      nloops * loop_layout().total + a256(sizeof(MatrixRef) * kMaxMatrices) + a256(sizeof(Shared));
  if ((size_t)budget_bytes < fixed + (1u << 20)) return PL_EINVAL;  // no room for any indices
  Server* S = new Server();
  cudaGetDevice(&S->dev);
  S->nbins = api_num_bins();
  S->nloops = nloops;
  S->budget = (size_t)budget_bytes;
  S->fixed_bytes = fixed;
  if (S->nbins > kMaxBinsS) {
    delete S;
    return PL_ENOTSUP;
  }
  if (const char* wm = getenv("PL_SERVE_WAVE_MS")) S->wave_us = std::max(0.1, atof(wm)) * 1000.0;
  if (const char* os = getenv("PL_SERVE_OLDEST_SHARE"))
    S->oldest_share = std::min(1.0, std::max(0.05, atof(os)));
  if (const char* im = getenv("PL_SERVE_IDLE_MS")) S->idle_ms = std::min(10000.0, std::max(0.05, atof(im)));
  const size_t arena = (size_t)budget_bytes - fixed;
  cudaError_t e;
  if ((e = cudaMalloc(&S->d_arena, arena)) != cudaSuccess ||
      (e = cudaMalloc(&S->d_mats, sizeof(MatrixRef) * kMaxMatrices)) != cudaSuccess ||
      (e = cudaMalloc(&S->sh, sizeof(Shared))) != cudaSuccess ||
      (e = cudaMemset(S->sh, 0, sizeof(Shared))) != cudaSuccess ||
      (e = cudaHostAlloc(&S->ctl, sizeof(Ctl), cudaHostAllocMapped)) != cudaSuccess ||
      (e = cudaHostAlloc(&S->ring, sizeof(RingDesc) * kRing, cudaHostAllocMapped)) != cudaSuccess ||
      (e = cudaHostAlloc(&S->h_pool, (size_t)host_pool_bytes, cudaHostAllocMapped)) != cudaSuccess ||
      (e = cudaHostGetDevicePointer((void**)&S->d_pool, S->h_pool, 0)) != cudaSuccess ||
      (e = cudaHostGetDevicePointer((void**)&S->ctl_d, S->ctl, 0)) != cudaSuccess ||
      (e = cudaHostGetDevicePointer((void**)&S->ring_d, S->ring, 0)) != cudaSuccess) {
    destroy(S);
    return cuda_fail(e);
  }
  memset(S->ctl, 0, sizeof(Ctl));
  for (int i = 0; i < kSlots; ++i) S->ctl->done_id[i] = -1;
  for (int i = kSlots - 1; i >= 0; --i) S->free_slots.push_back(i);
  S->arena.init(arena);
  S->pool.init((size_t)host_pool_bytes);
  if ((e = cudaStreamCreateWithFlags(&S->up, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&S->up_ev, cudaEventDisableTiming)) != cudaSuccess) {
    destroy(S);
    return cuda_fail(e);
  }
  for (int li = 0; li < nloops; ++li) {
    const int rc = build_loop(*S, S->loops[li], li);
    if (rc) {
      destroy(S);
      return rc;
    }
  }
  S->th = std::thread(scheduler, S);
  *server = S;
  return PL_OK;
}

int pl_serve_add_matrix(void* server, const float* A, int n, long long lda, int* matrix_id) {
  Server* S = (Server*)server;
  if (!S || !A || n < 1 || lda < n || !matrix_id) return PL_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  if ((int)S->mats.size() >= kMaxMatrices) return PL_ENOTSUP;
  const MatrixRef r{A, lda, n};
  const int id = (int)S->mats.size();
  // entries are appended and written before any request can name them
  cudaError_t e = cudaMemcpy(S->d_mats + id, &r, sizeof r, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e);
  S->mats.push_back(r);
  *matrix_id = id;
  return PL_OK;
}

int pl_serve_submit(void* server, int matrix_id, const int* idx, long long nsets, int k,
                    long long* request_id) {
  Server* S = (Server*)server;
  if (!S || !request_id || nsets < 1 || (!idx)) return PL_EINVAL;
  std::unique_lock<std::mutex> lk(S->mu);
  if (matrix_id < 0 || matrix_id >= (int)S->mats.size()) return PL_EINVAL;
  if (k < 1 || k > PL_KMAX || k > S->mats[matrix_id].n) return PL_EINVAL;
  if (req_dev_bytes(nsets, k) > S->arena.size) return PL_EINVAL;  // never admissible
  const size_t hb = req_host_bytes(nsets, k);
  if (hb > S->pool.size) return PL_EINVAL;
  size_t hoff = 0;
  if (!S->pool.alloc(hb, &hoff)) return PL_EBUSY;  // pinned pool full: retry later
  Request* r = new Request();
  r->id = S->next_id++;
  r->mat = matrix_id;
  r->k = k;
  r->nsets = nsets;
  r->host_off = hoff;
  r->host_len = hb;
  char* hp = S->h_pool + hoff;
  r->h_idx = (int*)hp;
  r->h_res = (double*)(hp + a256(sizeof(int) * (size_t)nsets * k));
  r->h_err = (int*)((char*)r->h_res + a256(3 * sizeof(double) * (size_t)nsets));
  r->t_submit = now_s();
  lk.unlock();
  memcpy(r->h_idx, idx, sizeof(int) * (size_t)nsets * k);
  lk.lock();
  S->reqs[r->id] = r;
  S->pending.push_back(r);
  *request_id = r->id;
  lk.unlock();
  S->cv_work.notify_one();
  return PL_OK;
}

int pl_serve_wait(void* server, long long request_id, double timeout_s, double* lmin, double* lmax,
                  double* delta, int* err, double* latency_s) {
  Server* S = (Server*)server;
  if (!S) return PL_EINVAL;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(request_id);
  if (it == S->reqs.end()) return PL_EINVAL;
  Request* r = it->second;
  const auto deadline = std::chrono::steady_clock::now() +
                        std::chrono::microseconds((long long)(std::max(timeout_s, 0.0) * 1e6));
  while (r->state != DONE && r->state != FAILED) {
    if (S->cv_done.wait_until(lk, deadline) == std::cv_status::timeout &&
        r->state != DONE && r->state != FAILED)
      return PL_ETIMEDOUT;
  }
  const int st = r->state == DONE ? PL_OK : r->status;
  if (st == PL_OK) {
    if (lmin) memcpy(lmin, r->h_res, sizeof(double) * (size_t)r->nsets);
    if (lmax) memcpy(lmax, r->h_res + r->nsets, sizeof(double) * (size_t)r->nsets);
    if (delta) memcpy(delta, r->h_res + 2 * r->nsets, sizeof(double) * (size_t)r->nsets);
    if (err) memcpy(err, r->h_err, sizeof(int) * (size_t)r->nsets);
  }
  if (latency_s) *latency_s = r->t_done - r->t_submit;
  S->pool.release(r->host_off, r->host_len);
  S->reqs.erase(it);
  delete r;
  return st;
}

int pl_serve_stats(void* server, double* out, int nout) {
  Server* S = (Server*)server;
  if (!S || !out || nout < 1) return PL_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  std::vector<double> l = S->lat;
  std::sort(l.begin(), l.end());
  auto pct = [&](double p) {
    if (l.empty()) return 0.0;
    const size_t i = (size_t)std::min<double>((double)l.size() - 1, std::ceil(p * l.size()) - 1);
    return l[i];
  };
  double mean = 0;
  for (double x : l) mean += x;
  if (!l.empty()) mean /= (double)l.size();
  long long waves = 0, launches = 0, idle = 0;
  int running = 0;
  for (int li = 0; li < S->nloops; ++li) {
    const Loop& L = S->loops[li];
    waves += *(volatile long long*)&S->ctl->waves[li];
    launches += L.launches;
    idle += L.idle_exits;
    running += L.running ? 1 : 0;
  }
  const double v[16] = {(double)l.size(),
                        (double)S->sets_done,
                        pct(0.50),
                        pct(0.99),
                        mean,
                        l.empty() ? 0.0 : l.back(),
                        S->t_last > S->t_first ? S->t_last - S->t_first : 0.0,
                        (double)S->arena.peak,
                        (double)S->arena.size,
                        (double)waves,
                        (double)S->running_max,
                        (double)S->pending.size(),
                        (double)launches,
                        (double)idle,
                        (double)(S->fixed_bytes + S->arena.size),
                        (double)running};
  for (int i = 0; i < nout && i < 16; ++i) out[i] = v[i];
  return PL_OK;
}

int pl_serve_reset_stats(void* server) {
  Server* S = (Server*)server;
  if (!S) return PL_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  S->lat.clear();
  S->sets_done = 0;
  S->running_max = 0;
  S->t_first = S->t_last = 0;
  S->arena.peak = S->arena.used;
  return PL_OK;
}

int pl_serve_destroy(void* server) { return destroy((Server*)server); }

}  // extern "C"
