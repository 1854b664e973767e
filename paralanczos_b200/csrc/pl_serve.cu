// pl_serve.cu -- serving: continuous batching of subset-eigensolve requests.
//
// The reference has no serving layer: each calculate_subeigs* call
// (ParaLanczos.cu:1725-1863) uploads one matrix and one batch of sets,
// launches, copies back and resets the device.  Here a server keeps several
// matrices resident and solves requests -- (matrix, k, a batch of index sets)
// -- as they arrive:
//
//   * submit() copies the request's indices into a pinned host pool and
//     queues it (PL_EBUSY when the pool is full: back-pressure);
//   * a scheduler thread admits queued requests in arrival order while their
//     indices fit the HBM budget arena (uploaded at admission, resident until
//     the request completes);
//   * work runs in "waves": a CSR batch of pieces (consecutive sets of one
//     request) whose sets may name different matrices and k, binned by k on
//     the device and solved by the persistent per-bin kernels of the batched
//     form on the wave's own streams.  A wave is sized to about
//     PL_SERVE_WAVE_MS (default 20) ms of estimated GPU work: the oldest
//     unfinished request gets up to PL_SERVE_OLDEST_SHARE (default 0.9) of
//     it, then requests with the
//     least remaining work fill the rest, so a large request is split over
//     waves while small requests that arrive behind it go out in the next
//     wave instead of waiting for it to finish;
//   * up to `max_waves` waves are in flight at once, each with its own stream
//     set, staging and kernel scratch, so requests that arrive while others
//     run are admitted as memory and wave slots free up and their kernels
//     overlap on the GPU;
//   * a finished wave's results are copied to pinned host memory; a request
//     completes with its last piece (host timestamps give the latency from
//     submit to completion) and its arena block is freed.
// A set's result does not depend on what else is in its wave: each set is
// solved by the bin's kernel on its own data with a fixed reduction order.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <atomic>
#include <chrono>
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

namespace pl {
namespace serve {

constexpr int kMaxMatrices = 64;
constexpr int kMaxBinsS = 16;

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
  size_t largest() const {
    size_t m = 0;
    for (auto& kv : free_) m = std::max(m, kv.second);
    return m;
  }
};

enum ReqState { PENDING = 0, ADMITTED = 1, DONE = 2, FAILED = 3 };

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
  long long next = 0;               // first set not yet given to a wave
  long long done = 0;               // sets whose results are back
};

// Arena charge of one request: its indices, resident on the device from
// admission to completion.
size_t req_dev_bytes(long long nsets, int k) { return a256(sizeof(int) * (size_t)nsets * k); }
size_t req_host_bytes(long long nsets, int k) {
  return a256(sizeof(int) * (size_t)nsets * k) + a256(3 * sizeof(double) * (size_t)nsets) +
         a256(sizeof(int) * (size_t)nsets);
}

// Whole-GPU time of one set of size k (microseconds), from the batched
// kernels' B200 throughput at each bin's largest k, scaled by (k / kmax)^3
// inside a bin and never below the previous bin's figure.  Only used to size
// waves: a misestimate changes wave lengths, never results.
double set_cost_us(int k) {
  static const int kb[9] = {8, 16, 32, 64, 128, 192, 256, 384, 512};
  static const double tb[9] = {0.001, 0.003, 0.014, 0.10, 0.88, 8.3, 25.5, 92.0, 253.0};
  for (int b = 0; b < 9; ++b) {
    if (k <= kb[b]) {
      const double x = (double)k / kb[b];
      return std::max(tb[b] * x * x * x, b ? tb[b - 1] : 0.0);
    }
  }
  return tb[8];
}

constexpr long long kWaveSets = 1 << 16;  // sets one wave can hold
constexpr long long kWaveIdx = 1 << 24;   // indices one wave can hold (64 MiB)

struct Piece {
  Request* r;
  long long first, count;  // sets [first, first + count) of the request
};

struct Wave {
  cudaStream_t st = nullptr;
  cudaStream_t side[kMaxBinsS] = {};
  cudaEvent_t fork = nullptr, join[kMaxBinsS] = {}, done = nullptr;
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  // device staging of one wave: its pieces' indices gathered contiguously,
  // CSR offsets, matrix ids, results
  int* d_idx = nullptr;
  long long nidx = 0;
  long long* d_off = nullptr;
  int* d_mat = nullptr;
  double* d_res = nullptr;  // lmin, lmax, delta: kWaveSets each
  int* d_err = nullptr;
  // pinned staging
  long long* h_off = nullptr;
  int* h_mat = nullptr;
  double* h_res = nullptr;
  int* h_err = nullptr;
  bool busy = false;
  long long nsets = 0;
  std::vector<Piece> pieces;
};

struct Server {
  int dev = 0;
  int nbins = 0;
  Arena arena;  // device budget: indices of admitted requests
  char* d_arena = nullptr;
  Arena pool;   // pinned host staging
  char* h_pool = nullptr;
  MatrixRef* d_mats = nullptr;
  std::vector<MatrixRef> mats;
  std::vector<Wave> waves;
  cudaStream_t up = nullptr;   // index uploads at admission
  cudaEvent_t up_ev = nullptr;
  double wave_us = 20000.0;    // GPU work one wave is sized for
  double oldest_share = 0.9;   // part of a wave the oldest unfinished request may take
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> pending;  // submitted, not admitted (arrival order)
  std::vector<Request*> active;  // admitted, not complete (arrival order)
  std::unordered_map<long long, Request*> reqs;
  std::thread th;
  std::atomic<bool> stop{false};
  long long next_id = 1;
  // statistics
  std::vector<double> lat;
  long long sets_done = 0, waves_launched = 0;
  int inflight_max = 0;
  double t_first = 0, t_last = 0;
};

int cuda_fail(cudaError_t e) {
  api_note_cuda(e);
  return e == cudaErrorMemoryAllocation ? PL_ENOMEM : PL_ECUDA;
}

int wave_alloc(Wave& w) {
  const size_t n = (size_t)kWaveSets;
  cudaError_t e;
  if ((e = cudaMalloc(&w.d_idx, sizeof(int) * (size_t)kWaveIdx)) != cudaSuccess) return cuda_fail(e);
  if ((e = cudaMalloc(&w.d_off, sizeof(long long) * (n + 1))) != cudaSuccess) return cuda_fail(e);
  if ((e = cudaMalloc(&w.d_mat, sizeof(int) * n)) != cudaSuccess) return cuda_fail(e);
  if ((e = cudaMalloc(&w.d_res, 3 * sizeof(double) * n)) != cudaSuccess) return cuda_fail(e);
  if ((e = cudaMalloc(&w.d_err, sizeof(int) * n)) != cudaSuccess) return cuda_fail(e);
  if ((e = cudaHostAlloc(&w.h_off, sizeof(long long) * (n + 1), 0)) != cudaSuccess) return cuda_fail(e);
  if ((e = cudaHostAlloc(&w.h_mat, sizeof(int) * n, 0)) != cudaSuccess) return cuda_fail(e);
  if ((e = cudaHostAlloc(&w.h_res, 3 * sizeof(double) * n, 0)) != cudaSuccess) return cuda_fail(e);
  if ((e = cudaHostAlloc(&w.h_err, sizeof(int) * n, 0)) != cudaSuccess) return cuda_fail(e);
  return PL_OK;
}

int wave_scratch(Wave& w, long long nsets) {
  const size_t need = api_binned_scratch(nsets, PL_FORM_BATCHED, false);
  if (w.scratch_bytes >= need) return PL_OK;
  if (w.scratch) cudaFree(w.scratch);
  w.scratch = nullptr;
  w.scratch_bytes = 0;
  cudaError_t e = cudaMalloc(&w.scratch, need);
  if (e != cudaSuccess) return cuda_fail(e);
  w.scratch_bytes = need;
  return PL_OK;
}

// Pieces of the next wave (server lock held): the oldest unfinished request
// first gets up to oldest_share of the wave (no request waits forever), then
// requests in order of least remaining work fill the rest, so a small
// request arriving behind a large one finishes in the next wave while the
// large one advances a wave at a time.  Every piece has at least one set.
void form_wave(Server& S, Wave& w) {
  w.pieces.clear();
  w.nsets = 0;
  w.nidx = 0;
  double used = 0.0;
  auto take = [&](Request* r, double allow) {
    const long long avail = r->nsets - r->next;
    const long long room = std::min(kWaveSets - w.nsets, (kWaveIdx - w.nidx) / r->k);
    if (avail <= 0 || room <= 0) return;
    const double c = set_cost_us(r->k);
    long long n = (long long)std::floor(allow / c);
    n = std::max(1LL, std::min(n, std::min(avail, room)));
    if (!w.pieces.empty() && w.pieces.back().r == r && w.pieces.back().first + w.pieces.back().count == r->next)
      w.pieces.back().count += n;
    else
      w.pieces.push_back(Piece{r, r->next, n});
    r->next += n;
    w.nsets += n;
    w.nidx += n * r->k;
    used += n * c;
  };
  Request* oldest = nullptr;
  for (Request* r : S.active)
    if (r->next < r->nsets) {
      oldest = r;
      break;
    }
  if (!oldest) return;
  take(oldest, S.oldest_share * S.wave_us);
  std::vector<Request*> order;
  for (Request* r : S.active)
    if (r->next < r->nsets) order.push_back(r);
  std::stable_sort(order.begin(), order.end(), [](const Request* a, const Request* b) {
    return (a->nsets - a->next) * set_cost_us(a->k) < (b->nsets - b->next) * set_cost_us(b->k);
  });
  for (Request* r : order) {
    if (used >= S.wave_us || w.nsets >= kWaveSets || w.nidx >= kWaveIdx) break;
    take(r, S.wave_us - used);
  }
}

// Enqueue one wave (scheduler thread, server lock NOT held; m0 is any
// registered matrix, read under the lock).
int launch_wave(Server& S, Wave& w, MatrixRef m0) {
  const long long total = w.nsets;
  cudaError_t e = cudaSuccess;
  auto note = [&](cudaError_t x) {
    if (e == cudaSuccess && x != cudaSuccess) e = x;
  };
  note(cudaStreamWaitEvent(w.st, S.up_ev, 0));  // the pieces' indices are on the device
  long long s = 0, o = 0;
  for (const Piece& p : w.pieces) {
    const long long cnt = p.count * p.r->k;
    note(cudaMemcpyAsync(w.d_idx + o, S.d_arena + p.r->dev_off + sizeof(int) * (size_t)(p.first * p.r->k),
                         sizeof(int) * (size_t)cnt, cudaMemcpyDeviceToDevice, w.st));
    for (long long i = 0; i < p.count; ++i, ++s) {
      w.h_off[s] = o + i * p.r->k;
      w.h_mat[s] = p.r->mat;
    }
    o += cnt;
  }
  w.h_off[total] = o;
  note(cudaMemcpyAsync(w.d_off, w.h_off, sizeof(long long) * (size_t)(total + 1), cudaMemcpyHostToDevice, w.st));
  note(cudaMemcpyAsync(w.d_mat, w.h_mat, sizeof(int) * (size_t)total, cudaMemcpyHostToDevice, w.st));
  if (e != cudaSuccess) return cuda_fail(e);
  MatrixF32 M{m0.A, m0.lda, m0.n};
  M.mats = S.d_mats;
  M.mat_id = w.d_mat;
  const size_t n = (size_t)kWaveSets;
  SetOutputs out{w.d_res, w.d_res + n, w.d_res + 2 * n, w.d_err, nullptr, nullptr};
  int rc;
  {
    // kernel shapes (and so the scratch size) may be retuned between waves
    std::lock_guard<std::mutex> lk(api_mutex());
    rc = wave_scratch(w, total);
    if (!rc)
      rc = api_launch_binned(M, w.d_idx, w.d_off, total, PL_FORM_BATCHED, out, w.scratch, w.st,
                             w.side, w.fork, w.join);
  }
  if (rc) return rc;
  for (int q = 0; q < 3; ++q)
    note(cudaMemcpyAsync(w.h_res + q * n, w.d_res + q * n, sizeof(double) * (size_t)total,
                         cudaMemcpyDeviceToHost, w.st));
  note(cudaMemcpyAsync(w.h_err, w.d_err, sizeof(int) * (size_t)total, cudaMemcpyDeviceToHost, w.st));
  note(cudaEventRecord(w.done, w.st));
  if (e != cudaSuccess) return cuda_fail(e);
  return PL_OK;
}

// Results of a finished wave -> its requests (server lock held).  A request
// completes when its last piece is back; then its arena block is freed.
void finish_wave(Server& S, Wave& w, int status) {
  const double t = now_s();
  const size_t n = (size_t)kWaveSets;
  long long s = 0;
  for (const Piece& p : w.pieces) {
    Request* r = p.r;
    if (status == PL_OK) {
      const size_t bytes = sizeof(double) * (size_t)p.count;
      memcpy(r->h_res + p.first, w.h_res + s, bytes);
      memcpy(r->h_res + r->nsets + p.first, w.h_res + n + s, bytes);
      memcpy(r->h_res + 2 * r->nsets + p.first, w.h_res + 2 * n + s, bytes);
      memcpy(r->h_err + p.first, w.h_err + s, sizeof(int) * (size_t)p.count);
    } else if (r->status == PL_OK) {
      r->status = status;
    }
    s += p.count;
    r->done += p.count;
    if (r->done == r->nsets) {
      r->state = r->status == PL_OK ? DONE : FAILED;
      r->t_done = t;
      S.lat.push_back(t - r->t_submit);
      S.t_last = t;
      if (r->state == DONE) S.sets_done += r->nsets;
      S.arena.release(r->dev_off, r->dev_len);
      S.active.erase(std::find(S.active.begin(), S.active.end(), r));
    }
  }
  w.pieces.clear();
  w.busy = false;
}

void scheduler(Server* sp) {
  Server& S = *sp;
  cudaSetDevice(S.dev);
  std::unique_lock<std::mutex> lk(S.mu);
  while (!S.stop.load()) {
    bool progressed = false;
    // ---- completions
    int inflight = 0;
    for (Wave& w : S.waves) {
      if (!w.busy) continue;
      const cudaError_t q = cudaEventQuery(w.done);
      if (q == cudaSuccess) {
        finish_wave(S, w, PL_OK);
        progressed = true;
      } else if (q != cudaErrorNotReady) {
        api_note_cuda(q);
        finish_wave(S, w, PL_ECUDA);
        progressed = true;
      } else {
        ++inflight;
      }
    }
    if (progressed) S.cv_done.notify_all();
    // ---- admission: arrival order, while the indices fit the arena
    bool admitted = false;
    while (!S.pending.empty()) {
      Request* r = S.pending.front();
      size_t off = 0;
      const size_t b = req_dev_bytes(r->nsets, r->k);
      if (!S.arena.alloc(b, &off)) break;
      r->dev_off = off;
      r->dev_len = b;
      r->state = ADMITTED;
      cudaError_t e = cudaMemcpyAsync(S.d_arena + off, r->h_idx, sizeof(int) * (size_t)r->nsets * r->k,
                                      cudaMemcpyHostToDevice, S.up);
      if (e != cudaSuccess) api_note_cuda(e);
      S.pending.pop_front();
      S.active.push_back(r);
      admitted = true;
    }
    if (admitted) {
      cudaEventRecord(S.up_ev, S.up);
      if (S.t_first == 0) S.t_first = now_s();
      progressed = true;
    }
    // ---- a wave into a free slot
    Wave* free_w = nullptr;
    for (Wave& w : S.waves)
      if (!w.busy) {
        free_w = &w;
        break;
      }
    if (free_w) {
      Wave& w = *free_w;
      form_wave(S, w);
      if (!w.pieces.empty()) {
        w.busy = true;
        const MatrixRef m0 = S.mats[0];
        lk.unlock();
        const int rc = launch_wave(S, w, m0);
        lk.lock();
        ++S.waves_launched;
        if (rc) {
          // nothing of the wave is in flight past the failed call: drain it
          cudaStreamSynchronize(w.st);
          finish_wave(S, w, rc);
          S.cv_done.notify_all();
        } else {
          S.inflight_max = std::max(S.inflight_max, inflight + 1);
        }
        progressed = true;
      }
    }
    if (!progressed) {
      bool any_busy = false;
      for (Wave& w : S.waves) any_busy |= w.busy;
      if (any_busy) {
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
  for (Wave& w : S->waves) {
    if (w.st) cudaStreamSynchronize(w.st);
    for (int b = 0; b < S->nbins; ++b) {
      if (w.side[b]) cudaStreamDestroy(w.side[b]);
      if (w.join[b]) cudaEventDestroy(w.join[b]);
    }
    if (w.st) cudaStreamDestroy(w.st);
    if (w.fork) cudaEventDestroy(w.fork);
    if (w.done) cudaEventDestroy(w.done);
    if (w.scratch) cudaFree(w.scratch);
    cudaFree(w.d_idx);
    cudaFree(w.d_off);
    cudaFree(w.d_mat);
    cudaFree(w.d_res);
    cudaFree(w.d_err);
    cudaFreeHost(w.h_off);
    cudaFreeHost(w.h_mat);
    cudaFreeHost(w.h_res);
    cudaFreeHost(w.h_err);
  }
  if (S->up) cudaStreamSynchronize(S->up);
  if (S->up) cudaStreamDestroy(S->up);
  if (S->up_ev) cudaEventDestroy(S->up_ev);
  for (auto& kv : S->reqs) delete kv.second;
  if (S->d_arena) cudaFree(S->d_arena);
  if (S->d_mats) cudaFree(S->d_mats);
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
  Server* S = new Server();
  cudaGetDevice(&S->dev);
  S->nbins = api_num_bins();
  if (S->nbins > kMaxBinsS) {
    delete S;
    return PL_ENOTSUP;
  }
  cudaError_t e;
  if ((e = cudaMalloc(&S->d_arena, (size_t)budget_bytes)) != cudaSuccess ||
      (e = cudaMalloc(&S->d_mats, sizeof(MatrixRef) * kMaxMatrices)) != cudaSuccess ||
      (e = cudaHostAlloc(&S->h_pool, (size_t)host_pool_bytes, 0)) != cudaSuccess) {
    destroy(S);
    return cuda_fail(e);
  }
  S->arena.init((size_t)budget_bytes);
  S->pool.init((size_t)host_pool_bytes);
  if (const char* wm = getenv("PL_SERVE_WAVE_MS")) S->wave_us = std::max(0.1, atof(wm)) * 1000.0;
  if (const char* os = getenv("PL_SERVE_OLDEST_SHARE"))
    S->oldest_share = std::min(1.0, std::max(0.05, atof(os)));
  if ((e = cudaStreamCreateWithFlags(&S->up, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&S->up_ev, cudaEventDisableTiming)) != cudaSuccess) {
    destroy(S);
    return cuda_fail(e);
  }
  S->waves.resize(max_waves);
  for (Wave& w : S->waves) {
    if ((e = cudaStreamCreateWithFlags(&w.st, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&w.fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&w.done, cudaEventDisableTiming)) != cudaSuccess) {
      destroy(S);
      return cuda_fail(e);
    }
    for (int b = 0; b < S->nbins; ++b) {
      if ((e = cudaStreamCreateWithFlags(&w.side[b], cudaStreamNonBlocking)) != cudaSuccess ||
          (e = cudaEventCreateWithFlags(&w.join[b], cudaEventDisableTiming)) != cudaSuccess) {
        destroy(S);
        return cuda_fail(e);
      }
    }
    // staging and kernel scratch of a full wave up front: growing them later
    // frees memory, which waits for the device
    int rc = wave_alloc(w);
    if (!rc) {
      std::lock_guard<std::mutex> lk(api_mutex());
      rc = wave_scratch(w, kWaveSets);
    }
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
  const double v[12] = {(double)l.size(),
                        (double)S->sets_done,
                        pct(0.50),
                        pct(0.99),
                        mean,
                        l.empty() ? 0.0 : l.back(),
                        S->t_last > S->t_first ? S->t_last - S->t_first : 0.0,
                        (double)S->arena.peak,
                        (double)S->arena.size,
                        (double)S->waves_launched,
                        (double)S->inflight_max,
                        (double)S->pending.size()};
  for (int i = 0; i < nout && i < 12; ++i) out[i] = v[i];
  return PL_OK;
}

int pl_serve_reset_stats(void* server) {
  Server* S = (Server*)server;
  if (!S) return PL_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  S->lat.clear();
  S->sets_done = 0;
  S->waves_launched = 0;
  S->inflight_max = 0;
  S->t_first = S->t_last = 0;
  S->arena.peak = S->arena.used;
  return PL_OK;
}

int pl_serve_destroy(void* server) { return destroy((Server*)server); }

}  // extern "C"
