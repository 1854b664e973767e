// pl_serve_plan.cuh -- the serving loop's shared structures and its wave
// policy, as host-and-device code (the device request loop of pl_serve.cu
// runs it; a CPU test runs the same function on adversarial request tables).
#pragma once
#include <math.h>

namespace pl {
namespace serve {

constexpr int kSlots = 1024;              // requests active on one loop at once
constexpr long long kWaveSets = 1 << 16;  // sets one wave can hold
constexpr long long kWaveIdx = 1 << 22;   // indices one wave can hold (16 MiB)
constexpr int kMaxPieces = 2048;          // request pieces one wave can hold

// Whole-GPU time of one set of size k (microseconds), from the batched
// kernels' B200 throughput at each bin's largest k, scaled by (k / kmax)^3
// inside a bin and never below the previous bin's figure.  Only used to size
// waves: a misestimate changes wave lengths, never results.
__host__ __device__ inline double set_cost_us(int k) {
  const int kb[9] = {8, 16, 32, 64, 128, 192, 256, 384, 512};
  const double tb[9] = {0.001, 0.003, 0.014, 0.10, 0.88, 8.3, 25.5, 92.0, 253.0};
  for (int b = 0; b < 9; ++b) {
    if (k <= kb[b]) {
      const double x = (double)k / kb[b];
      const double c = tb[b] * x * x * x;
      const double lo = b ? tb[b - 1] : 0.0;
      return c > lo ? c : lo;
    }
  }
  return tb[8];
}

// One admitted request, published by the host into a loop's ring (mapped
// pinned memory): its indices are already in the device arena.
struct RingDesc {
  long long id, nsets, arena_off;  // arena_off: first index, in ints
  double *lmin, *lmax, *delta;     // device views of the request's pinned results
  int* err;
  int slot, mat, k, pad;
};

// A loop's control block (mapped pinned memory).
struct Ctl {
  long long tail;              // host: descriptors published
  long long head;              // device: descriptors absorbed
  long long waves;             // device: waves formed
  int stop;                    // host: 1 = leave the loop
  int status;                  // device: 1 running, 2 left idle, 3 left on stop
  long long done_id[kSlots];   // device: id of the request completed in a slot
};

// Device-side state of an active request.
struct DevReq {
  long long id, nsets, next, done, arena_off;
  double *lmin, *lmax, *delta;
  int* err;
  int mat, k;
};

struct Piece {
  long long first, count;  // sets [first, first + count) of the request
  long long set0, idx0;    // its first set and first index in the wave
  int slot, k;
};

// A loop's planning state (device memory).
struct Plan {
  long long head;   // ring entries absorbed
  long long nsets;  // sets of the current wave (read by the binned launch)
  int nact, npieces;
  int act[kSlots];  // slots with unfinished sets, in arrival order
  Piece pieces[kMaxPieces];
};

// The next wave over the active requests act[0..nact) (arrival order): the
// oldest unfinished request first, up to oldest_share of wave_us
// microseconds of estimated work, then the request with the least work left,
// again and again, until the wave holds wave_us of work or is full (sets,
// indices or pieces).  Advances each request's `next`; returns the number of
// pieces written, *nsets their sets.  Every pass adds a piece or ends the
// wave, so it ends after at most kMaxPieces passes.
__host__ __device__ inline int form_wave(DevReq* tab, const int* act, int nact, double wave_us,
                                         double oldest_share, Piece* pieces, long long* nsets) {
  double used = 0.0;
  long long ns = 0, ni = 0;
  int np = 0;
  auto take = [&](int slot, double allow) -> bool {
    DevReq& r = tab[slot];
    const long long avail = r.nsets - r.next;
    long long room = kWaveSets - ns;
    const long long iroom = (kWaveIdx - ni) / r.k;
    room = room < iroom ? room : iroom;
    if (avail <= 0 || room <= 0 || np >= kMaxPieces) return false;
    const double c = set_cost_us(r.k);
    long long m = (long long)floor(allow / c);
    m = m < avail ? m : avail;
    m = m < room ? m : room;
    m = m > 1 ? m : 1;
    pieces[np++] = Piece{r.next, m, ns, ni, slot, r.k};
    r.next += m;
    ns += m;
    ni += m * r.k;
    used += m * c;
    return true;
  };
  for (int i = 0; i < nact; ++i)
    if (tab[act[i]].next < tab[act[i]].nsets) {
      take(act[i], oldest_share * wave_us);
      break;
    }
  for (int pass = 0; pass < kMaxPieces && used < wave_us && ns < kWaveSets && ni < kWaveIdx; ++pass) {
    int best = -1;
    double bw = 0.0;
    for (int i = 0; i < nact; ++i) {
      const DevReq& r = tab[act[i]];
      if (r.next >= r.nsets) continue;
      const double w = (double)(r.nsets - r.next) * set_cost_us(r.k);
      if (best < 0 || w < bw) {
        best = act[i];
        bw = w;
      }
    }
    if (best < 0 || !take(best, wave_us - used)) break;  // nothing left, or the wave is full
  }
  *nsets = ns;
  return np;
}

}  // namespace serve
}  // namespace pl
