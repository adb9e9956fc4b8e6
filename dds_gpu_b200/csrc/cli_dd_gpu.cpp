// dd_gpu: batch solver command line over libddg.so, with the reference's conventions
// (gpu/gpu_main.cu:1-6, 165-342):
//   dd_gpu K DEALS [TT_LOG2] [CHECK]        seeded random K-card deals (K = 13: full deals)
//   dd_gpu FILE.npy START DEALS [TT_LOG2]   Pgx DDS deals, checked against the file's tables
// Env: THREADS (solver lanes; default: fill the GPU), TIME_LIMIT (seconds; unfinished
// results are skipped in the check), PER_LEAD=1 (one job per lead instead of per strain),
// SEED (deal seed, default 12345), DEVICE. WAVE, STACK_KB and CHEAP_LOOP of the reference
// are accepted and ignored: there is only the wavefront kernel and it uses no call stack.
// CHECK (random mode, default 200): the first CHECK deals are solved again on the GPU with
// the other job split (per strain vs per lead) and a different TT size, an independent
// search whose tables must agree. Output: the reference's lines, last "N wrong of M
// checked"; exit 1 on a mismatch or an error, 2 on bad usage.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <string>
#include <vector>

#include "ddg.h"
#include "npy_pgx.hpp"

static int env_int(const char* name, int dflt) {
  const char* v = getenv(name);
  return v ? atoi(v) : dflt;
}

static int die(const char* what) {
  fprintf(stderr, "%s: %s\n", what, ddg_last_error());
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s K DEALS [TT_LOG2] [CHECK] | %s FILE.npy START DEALS [TT_LOG2]\n", argv[0], argv[0]);
    return 2;
  }
  bool file_mode = strstr(argv[1], ".npy") != nullptr;
  std::vector<uint64_t> hands;
  std::vector<uint8_t> want;
  long n;
  int tt_log2, check = 0;
  if (file_mode) {
    if (argc < 4) {
      fprintf(stderr, "usage: %s FILE.npy START DEALS [TT_LOG2]\n", argv[0]);
      return 2;
    }
    long start = atol(argv[2]);
    n = atol(argv[3]);
    tt_log2 = argc > 4 ? atoi(argv[4]) : 10;
    std::string err;
    if (!pgx::load(argv[1], start, n, hands, want, err)) {
      fprintf(stderr, "cannot load %s: %s\n", argv[1], err.c_str());
      return 1;
    }
  } else {
    int k = atoi(argv[1]);
    n = atol(argv[2]);
    tt_log2 = argc > 3 ? atoi(argv[3]) : 10;
    check = argc > 4 ? atoi(argv[4]) : 200;
    if (k < 1 || k > 13 || n < 0) {
      fprintf(stderr, "K must be 1..13 and DEALS >= 0\n");
      return 2;
    }
    hands.resize((size_t)n * 4);
    ddg_make_deals((uint64_t)env_int("SEED", 12345), 0, n, k, hands.data());
  }
  if (tt_log2 < 9) {
    fprintf(stderr, "TT_LOG2 must be >= 9\n");
    return 2;
  }
  ddg_config cfg;
  ddg_config_default(&cfg);
  cfg.tt_log2 = tt_log2;
  cfg.lanes = env_int("THREADS", 0);
  cfg.jobs_per_deal = env_int("PER_LEAD", 0) ? 20 : 5;
  cfg.device = env_int("DEVICE", 0);
  cfg.time_limit_s = getenv("TIME_LIMIT") ? atof(getenv("TIME_LIMIT")) : 0;
  if (cfg.lanes > 0) cfg.lanes = (cfg.lanes + cfg.block - 1) / cfg.block * cfg.block;  // whole blocks
  ddg_solver* s = nullptr;
  if (ddg_solver_create(&cfg, &s)) return die("solver");
  long jobs = n * cfg.jobs_per_deal;
  printf("%d threads, %ld deals, %ld solves, TT %.0f KB/solve, %.2f GB total\n", ddg_solver_lanes(s), n, jobs,
         (320 << tt_log2) / 1024.0, ddg_solver_bytes(s) / 1e9);
  std::vector<uint8_t> got((size_t)n * 20);
  ddg_stats st;
  auto t0 = std::chrono::steady_clock::now();
  if (ddg_solve_batch(s, hands.data(), n, got.data(), &st)) return die("solve");
  double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  printf("finished jobs: %lld in %.1f s = %.1f full-job deals/s\n", (long long)st.jobs_done, sec,
         st.jobs_done / (double)cfg.jobs_per_deal / sec);
  printf("GPU: %.3fs, %.0f deals/s (%.0f strain-solves/s), %.0f nodes/solve\n", sec, n / sec, n * 5 / sec,
         (double)st.nodes / (n * 5 > 0 ? n * 5 : 1));
  long bad = 0, checked = 0;
  if (file_mode) {
    for (long i = 0; i < n * 20; i++) {
      if (got[i] == 255) continue;
      bad += got[i] != want[i];
      checked++;
    }
  } else if (check > 0 && n > 0) {
    long m = check < n ? check : n;
    ddg_config c2 = cfg;
    c2.jobs_per_deal = cfg.jobs_per_deal == 5 ? 20 : 5;
    c2.tt_log2 = tt_log2 == 10 ? 11 : 10;
    c2.time_limit_s = 0;
    c2.lanes = 0;
    ddg_solver_destroy(s);
    s = nullptr;
    if (ddg_solver_create(&c2, &s)) return die("check solver");
    std::vector<uint8_t> again((size_t)m * 20);
    auto c0 = std::chrono::steady_clock::now();
    if (ddg_solve_batch(s, hands.data(), m, again.data(), nullptr)) return die("check solve");
    double cs = std::chrono::duration<double>(std::chrono::steady_clock::now() - c0).count();
    printf("check (GPU, %s jobs, TT 2^%d): %.0f deals/s\n", c2.jobs_per_deal == 20 ? "per-lead" : "per-strain",
           c2.tt_log2, m / cs);
    for (long i = 0; i < m * 20; i++) {
      if (got[i] == 255) continue;
      bad += got[i] != again[i];
      checked++;
    }
  }
  ddg_solver_destroy(s);
  printf("%ld wrong of %ld checked\n", bad, checked);
  return bad != 0;
}
