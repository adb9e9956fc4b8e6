// Test infrastructure / CPU baseline only: the reference's CPU solve path timed over a
// window, the way the reference reports its headline number (finished (deal, strain) jobs
// per second while a large deal set is being solved, README "full-job deals/s").
//
//   cpu_window DEALS.bin TT_LOG2 THREADS SLICE_S SLICES
//
// DEALS.bin: 32-byte records (4 x uint64 hands N,E,S,W). THREADS threads take (deal,
// strain) jobs in order, one TT each (cpu/cpu_main.cpp:41-72). The main thread counts the
// jobs finished in each of SLICES slices of SLICE_S seconds, prints one JSON line and ends
// the process at once (jobs still running are not counted; a running reference solve
// cannot be interrupted, so the process exit is what bounds the run).
//
// Built twice: with -DWITH_REF against the reference's src/dd.h where it lies
// (oracle/build_ref.sh -> oracle/_ref/cpu_window), and against the C restatement
// (oracle/Makefile -> oracle/_build/cpu_window).
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <unistd.h>

#include <atomic>
#include <chrono>
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
int g_slices = 1;

void finished(unsigned long long nodes) {
  double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - g_t0).count();
  long k = (long)(el / g_slice);
  if (k < g_slices) {
    g_done[k]++;
    g_nodes[k] += nodes;
  }
}
}  // namespace

int main(int argc, char** argv) {
  if (argc < 6) {
    fprintf(stderr, "usage: %s DEALS.bin TT_LOG2 THREADS SLICE_S SLICES\n", argv[0]);
    return 2;
  }
  FILE* f = fopen(argv[1], "rb");
  if (!f) {
    fprintf(stderr, "cannot open %s\n", argv[1]);
    return 1;
  }
  std::vector<uint64_t> hands;
  uint64_t rec[4];
  while (fread(rec, 8, 4, f) == 4) hands.insert(hands.end(), rec, rec + 4);
  fclose(f);
  const long n = (long)hands.size() / 4;
  const int tt_log2 = atoi(argv[2]);
  int threads = atoi(argv[3]);
  if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
  g_slice = atof(argv[4]);
  g_slices = atoi(argv[5]);
  if (n <= 0 || tt_log2 < 9 || tt_log2 > 24 || g_slice <= 0 || g_slices < 1 || g_slices > 4096) return 2;
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
#ifdef WITH_REF
        uint64_t before = c.nodes;
        dd_solve_strain(c, hands.data() + (job / 5) * 4, (int)(job % 5), out4);
        finished(c.nodes - before);
#else
        finished((unsigned long long)ddo_ctx_solve_strain(c, hands.data() + (job / 5) * 4, (int)(job % 5), out4));
#endif
      }
    }).detach();
  std::this_thread::sleep_until(g_t0 + std::chrono::duration<double>(g_slice * g_slices));
  printf("{\"threads\": %d, \"slice_s\": %g, \"jobs\": [", threads, g_slice);
  for (int k = 0; k < g_slices; k++) printf("%s%ld", k ? ", " : "", g_done[k].load());
  printf("], \"nodes\": [");
  for (int k = 0; k < g_slices; k++) printf("%s%llu", k ? ", " : "", g_nodes[k].load());
  printf("], \"kind\": \"%s\"}\n", 
#ifdef WITH_REF
         "reference"
#else
         "port"
#endif
  );
  fflush(stdout);
  _exit(0);
}
