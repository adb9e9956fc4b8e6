// dd_stream: streaming solver command line over libddg.so's streams, with the reference's
// conventions (gpu/stream_main.cu:1-12, 189-345):
//   dd_stream < deals.bin > results.bin
//       32-byte deals on stdin (4 x uint64 hands N,E,S,W); one 28-byte record per deal on
//       stdout as soon as it is solved, out of order: uint64 0-based input index + 20 bytes
//       tricks[strain C,D,H,S,NT][declarer N,E,S,W].
//   dd_stream bench SECONDS [TT_LOG2] [CHECK_EVERY] [RATE]
//       seeded random 13-card deals for SECONDS (RATE deals/s Poisson arrivals, 0 = as fast
//       as admitted), deals/s every 10 s, then throughput and p50/p99/p99.9 latency (arrival
//       to result on the host); every CHECK_EVERY-th solved deal is solved again afterwards
//       by a batch solve with the other job split and TT size (a GPU differential check).
// Env: THREADS (solver lanes; default: fill the GPU), PER_LEAD=1, SLOTS (ring, default
// 65536), SEED, DEVICE, TT_LOG2 (stdin mode). Summary lines go to stderr; exit 1 on an
// error or a wrong check.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <random>
#include <thread>
#include <vector>

#include "ddg.h"

using Clock = std::chrono::steady_clock;

static int env_int(const char* name, int dflt) {
  const char* v = getenv(name);
  return v ? atoi(v) : dflt;
}

static int die(const char* what) {
  fprintf(stderr, "%s: %s\n", what, ddg_last_error());
  return 1;
}

static double pct(std::vector<double>& v, double p) {
  if (v.empty()) return 0;
  size_t k = (size_t)(p * (v.size() - 1));
  std::nth_element(v.begin(), v.begin() + k, v.end());
  return v[k];
}

int main(int argc, char** argv) {
  const bool bench = argc > 1 && strcmp(argv[1], "bench") == 0;
  if (argc > 1 && !bench) {
    fprintf(stderr, "usage: %s < deals.bin > results.bin | %s bench SECONDS [TT_LOG2] [CHECK_EVERY] [RATE]\n",
            argv[0], argv[0]);
    return 2;
  }
  const double seconds = bench && argc > 2 ? atof(argv[2]) : 0;
  const int tt_log2 = bench ? (argc > 3 ? atoi(argv[3]) : 10) : env_int("TT_LOG2", 10);
  const long check_every = bench && argc > 4 ? atol(argv[4]) : 0;
  const double rate = bench && argc > 5 ? atof(argv[5]) : 0;
  if (bench && seconds <= 0) {
    fprintf(stderr, "SECONDS must be > 0\n");
    return 2;
  }
  std::vector<uint64_t> input;
  if (!bench) {
    uint64_t rec[4];
    while (fread(rec, 8, 4, stdin) == 4) input.insert(input.end(), rec, rec + 4);
  }
  ddg_config cfg;
  ddg_config_default(&cfg);
  cfg.tt_log2 = tt_log2;
  cfg.lanes = env_int("THREADS", 0);
  cfg.jobs_per_deal = env_int("PER_LEAD", 0) ? 20 : 5;
  cfg.device = env_int("DEVICE", 0);
  if (cfg.lanes > 0) cfg.lanes = (cfg.lanes + cfg.block - 1) / cfg.block * cfg.block;
  ddg_solver* s = nullptr;
  if (ddg_solver_create(&cfg, &s)) return die("solver");
  ddg_stream* st = nullptr;
  if (ddg_stream_open(s, env_int("SLOTS", 65536), 30.0, &st)) return die("stream");
  fprintf(stderr, "%d lanes, TT %.2f GB, %d jobs per deal, admission %lld deals in flight\n", ddg_solver_lanes(s),
          ddg_solver_bytes(s) / 1e9, cfg.jobs_per_deal, (long long)ddg_stream_capacity(st));

  const uint64_t seed = (uint64_t)env_int("SEED", 2026);
  std::vector<double> arrival, latency;
  std::vector<uint64_t> deals;  // every submitted deal (bench: generated as needed)
  std::vector<uint8_t> tables;
  std::vector<uint8_t> rec(65536 * 28);
  std::mt19937_64 rng(seed);
  std::exponential_distribution<double> gap(rate > 0 ? rate : 1.0);
  const auto t0 = Clock::now();
  auto last = t0;
  long long produced = 0, submitted = 0, solved = 0, last_solved = 0;
  double next_arrival = 0;
  const long long total = bench ? -1 : (long long)input.size() / 4;
  for (;;) {
    const double el = std::chrono::duration<double>(Clock::now() - t0).count();
    // Arrivals: stdin deals are all there at t = 0; bench deals arrive at RATE (or as fast
    // as the stream admits them).
    if (bench) {
      if (el < seconds) {
        while ((rate <= 0 && produced - submitted < 4096) || (rate > 0 && next_arrival <= el)) {
          deals.resize((size_t)(produced + 1) * 4);
          ddg_make_deals(seed, produced, 1, 13, deals.data() + produced * 4);
          arrival.push_back(rate > 0 ? next_arrival : el);
          produced++;
          if (rate > 0) next_arrival += gap(rng);
        }
      }
    } else if (produced == 0) {
      deals = input;
      produced = total;
      arrival.assign((size_t)total, 0.0);
    }
    if (submitted < produced) {
      int64_t acc = 0;
      if (ddg_stream_submit(st, deals.data() + submitted * 4, produced - submitted, &acc)) return die("submit");
      submitted += acc;
    }
    int64_t got = 0;
    if (ddg_stream_poll(st, rec.data(), 65536, &got)) return die("poll");
    const double now = std::chrono::duration<double>(Clock::now() - t0).count();
    for (int64_t k = 0; k < got; k++) {
      uint64_t idx;
      memcpy(&idx, rec.data() + k * 28, 8);
      latency.push_back(now - arrival[idx]);
      if (!bench) {
        fwrite(rec.data() + k * 28, 1, 28, stdout);
      } else if (check_every > 0 && idx % (uint64_t)check_every == 0) {
        tables.insert(tables.end(), rec.data() + k * 28, rec.data() + k * 28 + 28);
      }
    }
    solved += got;
    if (bench && std::chrono::duration<double>(Clock::now() - last).count() >= 10) {
      const double dt = std::chrono::duration<double>(Clock::now() - last).count();
      fprintf(stderr, "  %.0fs: %lld deals solved, last 10 s: %.1f deals/s, in flight %lld\n", now, solved,
              (solved - last_solved) / dt, (long long)ddg_stream_in_flight(st));
      last = Clock::now();
      last_solved = solved;
    }
    if (bench && now >= seconds) break;
    if (!bench && solved >= total) break;
    if (!got) std::this_thread::sleep_for(std::chrono::microseconds(200));
  }
  const double el = std::chrono::duration<double>(Clock::now() - t0).count();
  ddg_stats stats;
  if (ddg_stream_close(st, bench ? 0 : 1, &stats)) return die("close");
  std::vector<double> lat = latency;
  fprintf(stderr, "%lld deals solved in %.1f s (%.1f deals/s), %.0f nodes/deal, latency ms p50 %.1f p99 %.1f p99.9 %.1f\n",
          solved, el, solved / el, solved ? (double)stats.nodes / solved : 0.0, 1e3 * pct(lat, 0.5),
          1e3 * pct(lat, 0.99), 1e3 * pct(lat, 0.999));
  long wrong = 0, checked = 0;
  if (bench && !tables.empty()) {
    const long m = (long)tables.size() / 28;
    std::vector<uint64_t> h((size_t)m * 4);
    for (long i = 0; i < m; i++) {
      uint64_t idx;
      memcpy(&idx, tables.data() + i * 28, 8);
      memcpy(h.data() + i * 4, deals.data() + idx * 4, 32);
    }
    ddg_solver_destroy(s);
    s = nullptr;
    ddg_config c2 = cfg;
    c2.jobs_per_deal = cfg.jobs_per_deal == 5 ? 20 : 5;
    c2.tt_log2 = tt_log2 == 10 ? 11 : 10;
    c2.lanes = 0;
    if (ddg_solver_create(&c2, &s)) return die("check solver");
    std::vector<uint8_t> again((size_t)m * 20);
    if (ddg_solve_batch(s, h.data(), m, again.data(), nullptr)) return die("check solve");
    for (long i = 0; i < m; i++)
      for (int b = 0; b < 20; b++) {
        wrong += tables[i * 28 + 8 + b] != again[i * 20 + b];
        checked++;
      }
    fprintf(stderr, "GPU check: %ld wrong of %ld checked\n", wrong, checked);
  }
  ddg_solver_destroy(s);
  return wrong != 0;
}
