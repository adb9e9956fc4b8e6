// Test infrastructure only: a C-ABI shim around the reference solver's own headers
// (src/dd.h, src/dd_wave.h, src/npy.h of hsperr/dds_gpu), compiled from where they lie by
// oracle/build_ref.sh into oracle/_ref/libddref.so. Nothing in the product links this; the
// tests use it to pin the C restatement (oracle/dd_oracle.c) and to make golden fixtures,
// and bench.py's reference arm times it as the reference CPU path.
//
// Every entry point calls the reference's functions unchanged:
//   ref_solve_batch        -> dd_solve_strain        (src/dd.h:926), thread pool as cpu/cpu_main.cpp:41-72
//   ref_solve_batch_guess  -> dd_solve_strain_guess  (src/dd.h:915)
//   ref_wave_batch         -> dd_wave_step           (src/dd_wave.h:69), as tests/wave_test.cpp:33-46
//   ref_pgx_load           -> pgx_load/pgx_hands/pgx_tricks (src/npy.h:15-63)
#include <atomic>
#include <thread>
#include <vector>

#include "dd_wave.h"
#include "npy.h"

extern "C" {

int ref_bucket_bytes(void) { return (int)sizeof(DDBucket); }

// n deals x 5 strains. out20[i*20 + strain*4 + declarer]; job_nodes[i*5 + strain] (optional).
int ref_solve_batch(const uint64_t* hands, long n, int tt_log2, int threads, int* out20,
                    uint64_t* job_nodes) {
  if (tt_log2 < DD_TT_MIN_LOG2 || tt_log2 > 24 || n < 0) return -1;
  if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
  std::atomic<long> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; t++)
    pool.emplace_back([&] {
      std::vector<DDBucket> tt((size_t)1 << tt_log2);
      DDCtx c{};
      c.tt = tt.data();
      c.tt_mask = (1u << tt_log2) - 1;
      for (long job; (job = next++) < n * 5;) {
        uint64_t before = c.nodes;
        dd_solve_strain(c, hands + (job / 5) * 4, (int)(job % 5), out20 + (job / 5) * 20 + (job % 5) * 4);
        if (job_nodes) job_nodes[job] = c.nodes - before;
      }
    });
  for (auto& th : pool) th.join();
  return 0;
}

// Same with NS-trick seeds ns20[i*20 + strain*4 + declarer] (dd_solve_strain_guess).
int ref_solve_batch_guess(const uint64_t* hands, long n, int tt_log2, int threads,
                          const int* ns20, int* out20, uint64_t* job_nodes) {
  if (tt_log2 < DD_TT_MIN_LOG2 || tt_log2 > 24 || n < 0) return -1;
  if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
  std::atomic<long> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; t++)
    pool.emplace_back([&] {
      std::vector<DDBucket> tt((size_t)1 << tt_log2);
      DDCtx c{};
      c.tt = tt.data();
      c.tt_mask = (1u << tt_log2) - 1;
      for (long job; (job = next++) < n * 5;) {
        uint64_t before = c.nodes;
        long i = job / 5;
        int st = (int)(job % 5);
        dd_solve_strain_guess(c, hands + i * 4, st, ns20 + i * 20 + st * 4, out20 + i * 20 + st * 4);
        if (job_nodes) job_nodes[job] = c.nodes - before;
      }
    });
  for (auto& th : pool) th.join();
  return 0;
}

// The stage machine on one thread with jpd jobs per deal (5 or 20); job_nodes has n*jpd
// entries; steps[0..4] (optional) counts JOB, ROOT, ENTER, NEXT, RET steps.
int ref_wave_batch(const uint64_t* hands, long n, int tt_log2, int jpd, int* out20,
                   uint64_t* job_nodes, uint64_t* steps) {
  if (tt_log2 < DD_TT_MIN_LOG2 || tt_log2 > 24 || (jpd != 5 && jpd != 20)) return -1;
  std::vector<DDBucket> tt((size_t)1 << tt_log2);
  DDWave* w = new DDWave();
  w->c.tt = tt.data();
  w->c.tt_mask = (1u << tt_log2) - 1;
  w->hands = hands;
  w->out = out20;
  w->ring = n;
  w->work = 0;
  w->jpd = jpd;
  w->jobs = n * jpd;
  w->stage = DD_S_JOB;
  long next = 0;
  uint64_t mark = 0;
  long cur = -1;
  while (w->stage != DD_S_EXIT) {
    if (steps && w->stage < 5) steps[w->stage]++;
    int before = w->stage;
    if (before == DD_S_JOB) {  // the previous job (if any) has just finished
      if (cur >= 0 && job_nodes) job_nodes[cur] = w->c.nodes - mark;
      mark = w->c.nodes;
    }
    dd_wave_step(*w, [&] { return next++; });
    if (before == DD_S_JOB && w->stage != DD_S_EXIT) cur = w->job;
  }
  delete w;
  return 0;
}

// Number of deals in a Pgx .npy file, or -1.
long ref_pgx_count(const char* path) {
  PgxDeals d;
  if (!pgx_load(path, 0, 0, &d)) return -1;
  FILE* f = fopen(path, "rb");
  if (!f) return -1;
  char hdr[256] = {0};
  size_t got = fread(hdr, 1, sizeof(hdr) - 1, f);
  fclose(f);
  hdr[got] = 0;
  const char* sh = strstr(hdr + 10, "'shape': (2, ");
  return sh ? atol(sh + 13) : -1;
}

// Deals [start, start+count): hands (4 per deal) and the stored DDS tables, tricks20[i*20 +
// strain*4 + declarer].
int ref_pgx_load(const char* path, long start, long count, uint64_t* hands, int* tricks20) {
  PgxDeals d;
  if (!pgx_load(path, start, count, &d)) return -1;
  for (long i = 0; i < count; i++) {
    pgx_hands(d, i, hands + i * 4);
    for (int st = 0; st < 5; st++)
      for (int seat = 0; seat < 4; seat++) tricks20[i * 20 + st * 4 + seat] = pgx_tricks(d, i, seat, st);
  }
  return 0;
}

}  // extern "C"
