// Host-side check of the serving loop's wave policy (pl_serve_plan.cuh): the
// same form_wave the device planning kernel runs, driven wave after wave over
// request tables, with its invariants checked.  Built and run by
// tests/test_serve_plan.py (host code only: needs nvcc, no GPU).
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

// Runs waves until every set is scheduled; returns the number of waves, or a
// negative code on a broken invariant.
static long long drive(std::vector<DevReq>& tab, std::vector<int>& act, double wave_us, double share) {
  std::vector<Piece> pieces(kMaxPieces);
  std::vector<long long> seen(tab.size(), 0);
  long long waves = 0;
  for (;;) {
    bool work = false;
    for (int s : act) work |= tab[s].next < tab[s].nsets;
    if (!work) break;
    long long ns = 0;
    const int np = form_wave(tab.data(), act.data(), (int)act.size(), wave_us, share, pieces.data(), &ns);
    ++waves;
    if (np < 1 || np > kMaxPieces) return -1;          // no progress / overflow
    if (ns < 1 || ns > kWaveSets) return -2;
    long long set0 = 0, idx0 = 0;
    for (int p = 0; p < np; ++p) {
      const Piece& pc = pieces[p];
      if (pc.count < 1 || pc.set0 != set0 || pc.idx0 != idx0) return -3;  // contiguous wave layout
      if (pc.first != seen[pc.slot]) return -4;                           // request order, no gap/overlap
      seen[pc.slot] += pc.count;
      set0 += pc.count;
      idx0 += pc.count * pc.k;
    }
    if (set0 != ns || idx0 > kWaveIdx) return -5;
    if (waves > 10000000) return -6;
  }
  for (size_t s = 0; s < tab.size(); ++s)
    if (seen[s] != tab[s].nsets) return -7;             // every set exactly once
  return waves;
}

static DevReq req(long long nsets, int k) {
  DevReq r{};
  r.nsets = nsets;
  r.k = k;
  return r;
}

int main() {
  int fails = 0;
  // 1. indices fill the wave before the time budget: two large k = 100 requests
  //    (the case where a full wave must end the selection)
  {
    std::vector<DevReq> tab = {req(228000, 100), req(228000, 100)};
    std::vector<int> act = {0, 1};
    const long long w = drive(tab, act, 20000.0, 0.9);
    printf("index-full waves: %lld\n", w);
    fails += w <= 0;
  }
  // 2. sets fill the wave: many tiny sets
  {
    std::vector<DevReq> tab = {req(300000, 8), req(5, 8)};
    std::vector<int> act = {0, 1};
    const long long w = drive(tab, act, 20000.0, 0.9);
    printf("set-full waves: %lld\n", w);
    fails += w <= 0;
  }
  // 3. pieces fill the wave: more requests than pieces
  {
    std::vector<DevReq> tab;
    std::vector<int> act;
    for (int i = 0; i < kSlots; ++i) {
      tab.push_back(req(1 + i % 3, 8 + i % 7));
      act.push_back(i);
    }
    const long long w = drive(tab, act, 1e9, 0.9);
    printf("piece-full waves: %lld\n", w);
    fails += w <= 0;
  }
  // 4. random tables, short and long waves, every share
  for (int t = 0; t < 300; ++t) {
    const int n = 1 + (int)(next_rand() % 200);
    std::vector<DevReq> tab;
    std::vector<int> act;
    for (int i = 0; i < n; ++i) {
      const int k = 1 + (int)(next_rand() % 512);
      const long long ns = 1 + (long long)(next_rand() % 5000);
      tab.push_back(req(ns, k));
      act.push_back(i);
    }
    const double wave = (t % 3 == 0) ? 50.0 : (t % 3 == 1) ? 20000.0 : 1e7;
    const double share = 0.05 + 0.95 * (double)(next_rand() % 1000) / 999.0;
    const long long w = drive(tab, act, wave, share);
    if (w <= 0) {
      printf("random table %d: invariant %lld broken\n", t, w);
      ++fails;
    }
  }
  printf("%s\n", fails ? "FAIL" : "OK");
  return fails ? 1 : 0;
}
