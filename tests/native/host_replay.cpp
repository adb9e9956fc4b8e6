// Test infrastructure: the product's stage machine (dds_gpu_b200/csrc/ddg_search.cuh)
// compiled for the host and stepped one lane at a time, as the reference's own host check
// of its stage machine does (tests/wave_test.cpp). It lets the CPU test suite compare the
// GPU code's logic (tricks and node counts) with the oracle without a GPU. It is never
// part of the product path.
#include <stdint.h>
#include <string.h>

#include <atomic>
#include <thread>
#include <vector>

#include "ddg_search.cuh"

using namespace ddg;

namespace {
struct HostEnv {
  const u64* hands;
  long long n_jobs;
  int jpd, mode;
  const int8_t* seeds;  // n*20 NS seeds, strain*4 + declarer
  int* out20;
  uint64_t* job_nodes;
  std::atomic<long long>* next;
  Frame stack[64];
  TTBucket* tt;
  u32 mask;
  u64 start_nodes;
  LaneStats st;
  LaneStats& stats() { return st; }

  bool take(Lane& L) {
    long long job = (*next)++;
    if (job >= n_jobs) return false;
    L.job = job;
    L.deal = job / jpd;
    int sub = (int)(job % jpd);
    for (int i = 0; i < 4; i++) L.p.h[i] = hands[L.deal * 4 + i];
    L.strain = jpd == 5 ? sub : sub / 4;
    L.decl = jpd == 5 ? 0 : sub % 4;
    L.last_decl = jpd == 5 ? 3 : L.decl;
    L.mode = mode;
    start_nodes = st.nodes;
    return true;
  }
  int seed(const Lane& L) { return mode == MODE_STEP ? seeds[L.deal * 20 + L.strain * 4 + L.decl] : 7; }
  void answer(const Lane& L, int ns) {
    out20[L.deal * 20 + L.strain * 4 + L.decl] = (L.decl & 1) == 0 ? ns : 13 - ns;
  }
  void job_done(const Lane& L) {
    if (job_nodes) job_nodes[L.job] = st.nodes - start_nodes;
  }
};
}  // namespace

extern "C" {
// n deals, jpd 5 or 20 jobs per deal, mode 0 (binary search) / 1 (stepping from seeds).
// stats[0..4] = nodes, probes, hits, stores, TT bytes; stats[5..11] = enter exits.
int replay_solve(const uint64_t* hands, long long n, int tt_log2, int jpd, int mode,
                 const int8_t* seeds, int threads, int* out20, uint64_t* job_nodes,
                 uint64_t* stats) {
  if (tt_log2 < TT_MIN_LOG2 || tt_log2 > 22 || (jpd != 5 && jpd != 20)) return -1;
  if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
  std::atomic<long long> next{0};
  std::vector<std::thread> pool;
  std::vector<LaneStats> lane_stats(threads);
  for (int t = 0; t < threads; t++)
    pool.emplace_back([&, t] {
      std::vector<TTBucket> tt((size_t)1 << tt_log2);
      memset(tt.data(), 0, tt.size() * sizeof(TTBucket));
      HostEnv* env = new HostEnv();
      env->hands = hands;
      env->n_jobs = n * jpd;
      env->jpd = jpd;
      env->mode = mode;
      env->seeds = seeds;
      env->out20 = out20;
      env->job_nodes = job_nodes;
      env->next = &next;
      env->tt = tt.data();
      env->mask = (1u << tt_log2) - 1;
      memset(&env->st, 0, sizeof(env->st));
      Lane L;
      memset(&L, 0, sizeof(L));
      L.stage = ST_TAKE;
      while (L.stage != ST_IDLE) lane_step(L, *env);
      lane_stats[t] = env->st;
      delete env;
    });
  for (auto& th : pool) th.join();
  if (stats) {
    memset(stats, 0, 12 * sizeof(uint64_t));
    for (auto& s : lane_stats) {
      stats[0] += s.nodes;
      stats[1] += s.tt.probes;
      stats[2] += s.tt.hits;
      stats[3] += s.tt.stores;
      stats[4] += s.tt.bytes;
      for (int k = 0; k < 7; k++) stats[5 + k] += s.enter_exit[k];
    }
  }
  return 0;
}
}
