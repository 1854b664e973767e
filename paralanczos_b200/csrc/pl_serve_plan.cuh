// pl_serve_plan.cuh -- the serving loops' shared structures and their wave
// policy, as host-and-device code (the device request loops of pl_serve.cu
// run it; a CPU test runs the same function on adversarial request tables).
#pragma once
#include <math.h>

namespace pl {
namespace serve {

constexpr int kMaxLoops = 4;              // request loops (waves in flight) per server
constexpr int kSlots = 1024;              // requests active at once
constexpr long long kWaveSets = 1 << 16;  // sets one wave can hold
constexpr long long kWaveIdx = 1 << 22;   // indices one wave can hold (16 MiB)
constexpr int kMaxPieces = 2048;          // request pieces one wave can hold

// Whole-GPU time of one set of size k (microseconds), from the batched
// kernels' B200 throughput at each bin's largest k, scaled by (k / kmax)^3
// inside a bin and never below the previous bin's figure.  Only used to size
// waves: a misestimate changes wave lengths, never results.
__host__ __device__ inline double set_cost_us(int k) {
  const int kb[11] = {8, 16, 32, 48, 64, 96, 128, 192, 256, 384, 512};
  const double tb[11] = {0.001, 0.003, 0.0145, 0.045, 0.089, 0.334, 0.74, 3.2, 6.0, 38.9, 115.0};
  for (int b = 0; b < 11; ++b) {
    if (k <= kb[b]) {
      const double x = (double)k / kb[b];
      const double c = tb[b] * x * x * x;
      const double lo = b ? tb[b - 1] : 0.0;
      return c > lo ? c : lo;
    }
  }
  return tb[10];
}

// One admitted request, published by the host into the ring (mapped pinned
// memory): its indices are already in the device arena.
struct RingDesc {
  long long id, nsets, arena_off;  // arena_off: first index, in ints
  double *lmin, *lmax, *delta;     // device views of the request's pinned results
  int* err;
  int slot, mat, k, pad;
};

// The server's control block (mapped pinned memory).
struct Ctl {
  long long tail;                // host: descriptors published
  long long head;                // device: descriptors absorbed (a copy for the host)
  int stop;                      // host: 1 = the loops leave
  int pad;
  int status[kMaxLoops];         // device: 1 running, 2 left idle, 3 left on stop
  long long waves[kMaxLoops];    // device: waves formed by each loop
  long long done_id[kSlots];     // device: id of the request completed in a slot
};

// Device-side state of an active request, shared by every loop.  `next` (the
// first set no wave has claimed) only ever grows, by atomic claims; `live` is
// 1 from the request's absorption until its last set is done.
struct DevReq {
  long long id, nsets, next, done, arena_off;
  double *lmin, *lmax, *delta;
  int* err;
  int mat, k, live, pad;
};

// Device memory shared by the loops: the ring cursor and the request table.
struct Shared {
  unsigned long long head;  // ring entries claimed by an absorbing planner
  long long pad[15];
  DevReq tab[kSlots];
};

struct Piece {
  long long first, count;  // sets [first, first + count) of the request
  long long set0, idx0;    // its first set and first index in the wave
  int slot, k;
};

// One loop's current wave (device memory).
struct Plan {
  long long nsets;  // sets of the wave (read by the binned launch)
  int npieces, pad;
  Piece pieces[kMaxPieces];
};

// A request with sets left, as the planner saw it.
struct Cand {
  long long id, remaining;
  int slot, k;
};

// The next wave over the candidates: the oldest request first (lowest id), up
// to oldest_share of wave_us microseconds of estimated work, then the one with
// the least work left, again and again, until the wave holds wave_us of work
// or is full (sets, indices or pieces).  claim(slot, want, &first) takes up to
// `want` sets of a request for this wave and returns how many it got (fewer,
// or none, when other waves claimed them first).  Returns the number of
// pieces written, *nsets their sets.  Every pass adds a piece, empties a
// candidate or ends the wave, so it ends after kMaxPieces + nc passes at most.
template <class Claim>
__host__ __device__ inline int form_wave(Cand* c, int nc, double wave_us, double oldest_share, Piece* pieces,
                                         long long* nsets, Claim claim) {
  double used = 0.0;
  long long ns = 0, ni = 0;
  int np = 0;
  // 1: a piece was added; 0: the candidate had nothing left; -1: wave full
  auto take = [&](Cand& x, double allow) -> int {
    long long room = kWaveSets - ns;
    const long long iroom = (kWaveIdx - ni) / x.k;
    room = room < iroom ? room : iroom;
    if (room <= 0 || np >= kMaxPieces) return -1;
    if (x.remaining <= 0) return 0;
    const double cst = set_cost_us(x.k);
    long long m = (long long)floor(allow / cst);
    m = m < x.remaining ? m : x.remaining;
    m = m < room ? m : room;
    m = m > 1 ? m : 1;
    long long first = 0;
    const long long got = claim(x.slot, m, &first);
    if (got <= 0) {
      x.remaining = 0;
      return 0;
    }
    x.remaining = got < m ? 0 : x.remaining - got;
    pieces[np++] = Piece{first, got, ns, ni, x.slot, x.k};
    ns += got;
    ni += got * x.k;
    used += got * cst;
    return 1;
  };
  int oi = -1;
  for (int i = 0; i < nc; ++i)
    if (c[i].remaining > 0 && (oi < 0 || c[i].id < c[oi].id)) oi = i;
  if (oi >= 0) take(c[oi], oldest_share * wave_us);
  for (int pass = 0; pass < kMaxPieces + nc && used < wave_us && ns < kWaveSets && ni < kWaveIdx; ++pass) {
    int best = -1;
    double bw = 0.0;
    for (int i = 0; i < nc; ++i) {
      if (c[i].remaining <= 0) continue;
      const double w = (double)c[i].remaining * set_cost_us(c[i].k);
      if (best < 0 || w < bw || (w == bw && c[i].id < c[best].id)) {
        best = i;
        bw = w;
      }
    }
    if (best < 0 || take(c[best], wave_us - used) < 0) break;  // nothing left, or the wave is full
  }
  *nsets = ns;
  return np;
}

}  // namespace serve
}  // namespace pl
