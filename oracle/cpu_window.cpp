// Test infrastructure / CPU baseline only: the reference's CPU solve path timed over a
// window, the way the reference reports its headline number (finished (deal, strain) jobs
// per second while a large deal set is being solved, README "full-job deals/s"), with the
// search nodes of the window (the work rate) and the results of every finished job.
//
//   cpu_window SRC TT_LOG2 THREADS SLICE_S SLICES [WARMUP] [TABLES_OUT]
//
// SRC: a file of 32-byte records (4 x uint64 hands N,E,S,W), or gen:SEED:N:K for N seeded
// K-card deals made here (splitmix64 and a Fisher-Yates shuffle of the 52 cards, deal d from
// its own stream x = SEED ^ (0xD1B54A32D192ED03 * (d + 1)), cards 0..4K-1 of the shuffle
// round-robin to N,E,S,W), so a caller needs nothing of the product to make the deals.
// THREADS threads (0 = every host core) take (deal, strain) jobs in order, one TT each
// (cpu/cpu_main.cpp:41-72). The main thread counts the jobs finished and their search nodes
// in each of SLICES slices of SLICE_S seconds, prints one JSON line and ends the process at
// once (jobs still running are not counted; a running reference solve cannot be
// interrupted, so the process exit is what bounds the run). Jobs finished in slices WARMUP
// and later also give the p50 / p99 of their own search time (start to end, ms).
// TABLES_OUT (optional) receives N * 20 bytes, tricks[deal][strain][declarer] of every job
// finished inside the window, 255 elsewhere.
//
// Built twice: with -DWITH_REF against the reference's src/dd.h where it lies
// (oracle/build_ref.sh -> oracle/_ref/cpu_window), and against the C restatement
// (oracle/Makefile -> oracle/_build/cpu_window).
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <mutex>
#include <thread>
#include <vector>

#ifdef WITH_REF
#include "dd.h"
#else
extern "C" {
void* ddo_ctx_new(int tt_log2);
long long ddo_ctx_solve_strain(void* ctx, const uint64_t* hands4, int strain, int* out4);
void ddo_ctx_free(void* ctx);
}
#endif

namespace {
std::atomic<long> g_next{0};
std::atomic<long> g_done[4096];
std::atomic<unsigned long long> g_nodes[4096];
std::chrono::steady_clock::time_point g_t0;
double g_slice = 1.0;
int g_slices = 1, g_warmup = 0;
std::vector<uint8_t> g_tables;
std::mutex g_mu;
std::vector<double> g_lat_ms;  // search time of the jobs finished in the timed slices

double now_s() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - g_t0).count(); }

void finished(long job, const int* out4, unsigned long long nodes, double t_start) {
  const double el = now_s();
  const long k = (long)(el / g_slice);
  if (k >= g_slices) return;
  g_done[k]++;
  g_nodes[k] += nodes;
  for (int d = 0; d < 4; d++) g_tables[(job / 5) * 20 + (job % 5) * 4 + d] = (uint8_t)out4[d];
  if (k >= g_warmup) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_lat_ms.push_back(1e3 * (el - t_start));
  }
}

uint64_t splitmix_next(uint64_t& x) {
  x += 0x9E3779B97F4A7C15ull;
  uint64_t z = x;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

void make_deals(uint64_t seed, long n, int k, std::vector<uint64_t>& hands) {
  hands.assign((size_t)n * 4, 0);
  for (long d = 0; d < n; d++) {
    uint64_t x = seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(d + 1));
    int cards[52];
    for (int i = 0; i < 52; i++) cards[i] = (i / 13) * 16 + i % 13;
    for (int i = 51; i > 0; i--) {
      int j = (int)(splitmix_next(x) % (uint64_t)(i + 1));
      std::swap(cards[i], cards[j]);
    }
    for (int i = 0; i < 4 * k; i++) hands[d * 4 + i % 4] |= 1ull << cards[i];
  }
}

double pct(std::vector<double> v, double p) {
  if (v.empty()) return -1;
  size_t k = (size_t)(p * (double)(v.size() - 1));
  std::nth_element(v.begin(), v.begin() + k, v.end());
  return v[k];
}
}  // namespace

int main(int argc, char** argv) {
  if (argc < 6) {
    fprintf(stderr, "usage: %s DEALS.bin|gen:SEED:N:K TT_LOG2 THREADS SLICE_S SLICES [WARMUP] [TABLES_OUT]\n",
            argv[0]);
    return 2;
  }
  std::vector<uint64_t> hands;
  if (strncmp(argv[1], "gen:", 4) == 0) {
    unsigned long long seed = 0;
    long n = 0;
    int k = 0;
    if (sscanf(argv[1] + 4, "%llu:%ld:%d", &seed, &n, &k) != 3 || n <= 0 || k < 1 || k > 13) return 2;
    make_deals(seed, n, k, hands);
  } else {
    FILE* f = fopen(argv[1], "rb");
    if (!f) {
      fprintf(stderr, "cannot open %s\n", argv[1]);
      return 1;
    }
    uint64_t rec[4];
    while (fread(rec, 8, 4, f) == 4) hands.insert(hands.end(), rec, rec + 4);
    fclose(f);
  }
  const long n = (long)hands.size() / 4;
  const int tt_log2 = atoi(argv[2]);
  int threads = atoi(argv[3]);
  if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
  g_slice = atof(argv[4]);
  g_slices = atoi(argv[5]);
  g_warmup = argc > 6 ? atoi(argv[6]) : 0;
  const char* tables_out = argc > 7 ? argv[7] : nullptr;
  if (n <= 0 || tt_log2 < 9 || tt_log2 > 24 || g_slice <= 0 || g_slices < 1 || g_slices > 4096) return 2;
  g_tables.assign((size_t)n * 20, 255);
  g_t0 = std::chrono::steady_clock::now();
  for (int t = 0; t < threads; t++)
    std::thread([n, tt_log2, &hands] {
#ifdef WITH_REF
      std::vector<DDBucket> tt((size_t)1 << tt_log2);
      DDCtx c{};
      c.tt = tt.data();
      c.tt_mask = (1u << tt_log2) - 1;
#else
      void* c = ddo_ctx_new(tt_log2);
#endif
      int out4[4];
      for (long job; (job = g_next++) < n * 5;) {
        const double t_start = now_s();
#ifdef WITH_REF
        uint64_t before = c.nodes;
        dd_solve_strain(c, hands.data() + (job / 5) * 4, (int)(job % 5), out4);
        finished(job, out4, c.nodes - before, t_start);
#else
        unsigned long long nodes =
            (unsigned long long)ddo_ctx_solve_strain(c, hands.data() + (job / 5) * 4, (int)(job % 5), out4);
        finished(job, out4, nodes, t_start);
#endif
      }
    }).detach();
  std::this_thread::sleep_until(g_t0 + std::chrono::duration<double>(g_slice * g_slices));
  std::vector<double> lat;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    lat = g_lat_ms;
  }
  if (tables_out) {
    // A job finishing now may be writing its row; jobs finished inside the window wrote
    // theirs before they were counted.
    FILE* f = fopen(tables_out, "wb");
    if (!f || fwrite(g_tables.data(), 1, g_tables.size(), f) != g_tables.size()) {
      fprintf(stderr, "cannot write %s\n", tables_out);
      _exit(1);
    }
    fclose(f);
  }
  printf("{\"threads\": %d, \"slice_s\": %g, \"deals\": %ld, \"jobs\": [", threads, g_slice, n);
  for (int k = 0; k < g_slices; k++) printf("%s%ld", k ? ", " : "", g_done[k].load());
  printf("], \"nodes\": [");
  for (int k = 0; k < g_slices; k++) printf("%s%llu", k ? ", " : "", g_nodes[k].load());
  printf("], \"job_ms_p50\": %.3f, \"job_ms_p99\": %.3f, \"kind\": \"%s\"}\n", pct(lat, 0.5), pct(lat, 0.99),
#ifdef WITH_REF
         "reference"
#else
         "port"
#endif
  );
  fflush(stdout);
  _exit(0);
}
