// Host-side check of the serving loops' wave policy (pl_serve_plan.cuh): the
// same form_wave the device planning kernels run, driven wave after wave over
// request tables -- by one planner, and by two planners whose claims
// interleave the way two loops' atomic claims can -- with its invariants
// checked.  Built and run by tests/test_serve_plan.py (host code only: needs
// nvcc, no GPU).
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#include "../paralanczos_b200/csrc/pl_serve_plan.cuh"

using namespace pl::serve;

static unsigned long long rng = 88172645463325252ull;
static unsigned long long next_rand() {
  rng ^= rng << 13;
  rng ^= rng >> 7;
  rng ^= rng << 17;
  return rng;
}

struct Table {
  std::vector<long long> nsets, next, seen;
  std::vector<int> k;
};

// Candidates as a scan sees them (remaining = nsets - next; stale views are
// allowed: `lag` adds sets that another planner already claimed).
static int scan(const Table& T, std::vector<Cand>& c, long long lag) {
  int n = 0;
  for (size_t s = 0; s < T.nsets.size(); ++s)
    if (T.next[s] < T.nsets[s]) c[n++] = Cand{(long long)s, T.nsets[s] - T.next[s] + lag, (int)s, T.k[s]};
  return n;
}

// Checks one wave; returns 0 or a negative code.
static int check_wave(Table& T, const std::vector<Piece>& p, int np, long long ns) {
  if (np < 0 || np > kMaxPieces || ns < 0 || ns > kWaveSets) return -2;
  long long set0 = 0, idx0 = 0;
  for (int i = 0; i < np; ++i) {
    const Piece& pc = p[i];
    if (pc.count < 1 || pc.set0 != set0 || pc.idx0 != idx0) return -3;  // contiguous wave layout
    for (long long j = 0; j < pc.count; ++j)
      if (pc.first + j >= T.nsets[pc.slot]) return -4;                 // never past the request
    T.seen[pc.slot] += pc.count;
    set0 += pc.count;
    idx0 += pc.count * pc.k;
  }
  if (set0 != ns || idx0 > kWaveIdx) return -5;
  return 0;
}

// Waves by `planners` planners taking turns (their claims interleave) until
// every set is taken; returns the number of waves or a negative code.
static long long drive(Table& T, double wave_us, double share, int planners) {
  std::vector<Cand> c(T.nsets.size() + 1);
  std::vector<Piece> p(kMaxPieces);
  long long waves = 0;
  for (;;) {
    bool work = false;
    for (size_t s = 0; s < T.nsets.size(); ++s) work |= T.next[s] < T.nsets[s];
    if (!work) break;
    // each planner scans first (so later ones see stale counts), then claims
    std::vector<std::vector<Cand>> views(planners, c);
    std::vector<int> nc(planners);
    for (int q = 0; q < planners; ++q) nc[q] = scan(T, views[q], q ? 17 : 0);
    bool any = false;
    for (int q = 0; q < planners; ++q) {
      auto claim = [&](int slot, long long want, long long* first) -> long long {
        const long long old = T.next[slot];
        T.next[slot] += want;  // like atomicAdd: may pass nsets
        if (old >= T.nsets[slot]) return 0;
        *first = old;
        return want < T.nsets[slot] - old ? want : T.nsets[slot] - old;
      };
      long long ns = 0;
      const int np = form_wave(views[q].data(), nc[q], wave_us, share, p.data(), &ns, claim);
      ++waves;
      const int rc = check_wave(T, p, np, ns);
      if (rc) return rc;
      any |= np > 0;
    }
    if (!any) return -1;  // nobody made progress while work was left
    if (waves > 10000000) return -6;
  }
  for (size_t s = 0; s < T.nsets.size(); ++s)
    if (T.seen[s] != T.nsets[s]) return -7;  // every set exactly once
  return waves;
}

static Table table(const std::vector<long long>& ns, const std::vector<int>& k) {
  Table T;
  T.nsets = ns;
  T.k = k;
  T.next.assign(ns.size(), 0);
  T.seen.assign(ns.size(), 0);
  return T;
}

int main() {
  int fails = 0;
  for (int planners = 1; planners <= 3; ++planners) {
    // indices fill the wave before its time budget (two large k = 100 requests)
    {
      Table T = table({228000, 228000}, {100, 100});
      const long long w = drive(T, 20000.0, 0.9, planners);
      printf("planners %d index-full waves: %lld\n", planners, w);
      fails += w <= 0;
    }
    // sets fill the wave: many tiny sets
    {
      Table T = table({300000, 5}, {8, 8});
      const long long w = drive(T, 20000.0, 0.9, planners);
      printf("planners %d set-full waves: %lld\n", planners, w);
      fails += w <= 0;
    }
    // pieces fill the wave: more requests than pieces
    {
      std::vector<long long> ns;
      std::vector<int> k;
      for (int i = 0; i < kSlots; ++i) {
        ns.push_back(1 + i % 3);
        k.push_back(8 + i % 7);
      }
      Table T = table(ns, k);
      const long long w = drive(T, 1e9, 0.9, planners);
      printf("planners %d piece-full waves: %lld\n", planners, w);
      fails += w <= 0;
    }
    // random tables, short and long waves, every share
    for (int t = 0; t < 200; ++t) {
      const int n = 1 + (int)(next_rand() % 200);
      std::vector<long long> ns;
      std::vector<int> k;
      for (int i = 0; i < n; ++i) {
        k.push_back(1 + (int)(next_rand() % 512));
        ns.push_back(1 + (long long)(next_rand() % 5000));
      }
      Table T = table(ns, k);
      const double wave = (t % 3 == 0) ? 50.0 : (t % 3 == 1) ? 20000.0 : 1e7;
      const double share = 0.05 + 0.95 * (double)(next_rand() % 1000) / 999.0;
      const long long w = drive(T, wave, share, planners);
      if (w <= 0) {
        printf("planners %d random table %d: invariant %lld broken\n", planners, t, w);
        ++fails;
      }
    }
  }
  printf("%s\n", fails ? "FAIL" : "OK");
  return fails ? 1 : 0;
}
