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

#define DDG_EXIT_COUNTS 1  // the replay reports the ENTER outcomes
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
  Frame stack[STACK_DEPTH];
  TTBucket* tt;
  u32 mask;
  u64 start_nodes;
  LaneStats st;
  LaneStats& stats() { return st; }
  TaskPool* pool() { return nullptr; }
  bool want_donation() { return false; }
  void unreserve() {}
  int claim_start() { return 0; }
  u64 work_nodes() { return st.nodes - start_nodes; }
  void task_started() { start_nodes = st.nodes; }
  u64 tt_key_ = 0;
  u64& tt_key() { return tt_key_; }
  // Shared-TT helping (SimEnv overrides these; a lone lane has no helpers).
  bool share_tt() { return false; }
  TTBucket* tt_of(int) { return tt; }
  long long self() { return 0; }
  void tt_users_add(int, int) {}
  int tt_users(int) { return 0; }
  const int8_t* hints = nullptr;  // n*20 root leads to try first (the guide's), or null
  int root_hint(const Lane& L) { return hints ? (int)hints[L.deal * 20 + L.strain * 4 + L.decl] : -1; }
  int cheap_limit() { return 0; }
  bool fuse_follow() { return false; }
  void root_best(const Lane&, int) {}

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

// A block of lanes stepped through the GPU kernel's phases in order (one lane at a time),
// with the block's task pool: the helping logic (donation, retraction, merging,
// abandonment) runs exactly as on the GPU, deterministically.
struct SimShared {
  TaskPool pool;
  int budget = 0;  // donations allowed this iteration
  bool eager = false;
  int cheap_limit = 0;  // most cheap stages per lane per pass, as the GPU kernel's
  bool share = false;   // helpers search in their donor's TT
  std::vector<TTBucket*> tts;  // every lane's TT
  std::vector<int> users;      // helpers searching in each lane's TT
};
struct SimEnv : HostEnv {
  SimShared* sh;
  int lane_id = 0, min_nodes = 0;
  TaskPool* pool() { return &sh->pool; }
  bool share_tt() { return sh->share; }
  TTBucket* tt_of(int lane) { return sh->tts[lane]; }
  long long self() { return lane_id; }
  void tt_users_add(int lane, int d) { sh->users[lane] += d; }
  int tt_users(int lane) { return sh->users[lane]; }
  bool want_donation() {
    if (sh->budget <= 0 || (!sh->eager && sh->pool.queued >= sh->pool.hungry)) return false;
    sh->budget--;
    sh->pool.queued++;
    return true;
  }
  void unreserve() { sh->pool.queued--; }
  int claim_start() { return lane_id * 61; }
  int cheap_limit() { return sh->cheap_limit; }
  u64 work_nodes() { return st.nodes - start_nodes + (u64)DONATE_MIN_NODES - (u64)min_nodes; }
};


extern "C" {
// n deals on one simulated block of `lanes` lanes, with helping; `eager` donates whenever a
// lane could (not only when lanes are hungry). Results and nodes as replay_solve; stats[12]
// = tasks posted, stats[13] = block iterations. `share`: helpers search in their donor's TT.
int replay_block_ex(const uint64_t* hands, long long n, int tt_log2, int jpd, int lanes, int eager, int free_below,
                    int free_steps, int* out20, uint64_t* stats, int cheap_limit, int share);
int replay_block(const uint64_t* hands, long long n, int tt_log2, int jpd, int lanes, int eager, int free_below,
                 int free_steps, int* out20, uint64_t* stats, int cheap_limit) {
  return replay_block_ex(hands, n, tt_log2, jpd, lanes, eager, free_below, free_steps, out20, stats, cheap_limit, 0);
}
int replay_block_ex(const uint64_t* hands, long long n, int tt_log2, int jpd, int lanes, int eager, int free_below,
                    int free_steps, int* out20, uint64_t* stats, int cheap_limit, int share) {
  if (tt_log2 < TT_MIN_LOG2 || tt_log2 > 16 || (jpd != 5 && jpd != 20) || lanes < 1 || lanes > 1024) return -1;
  std::atomic<long long> next{0};
  SimShared* sh = new SimShared();
  sh->share = share != 0;
  sh->users.assign(lanes, 0);
  memset(&sh->pool, 0, sizeof(sh->pool));
  std::vector<SimEnv*> envs(lanes);
  std::vector<std::vector<TTBucket>> tts(lanes);
  std::vector<Lane> L(lanes);
  for (int i = 0; i < lanes; i++) {
    tts[i].assign((size_t)1 << tt_log2, TTBucket());
    memset(tts[i].data(), 0, tts[i].size() * sizeof(TTBucket));
    SimEnv* e = new SimEnv();
    e->hands = hands;
    e->n_jobs = n * jpd;
    e->jpd = jpd;
    e->mode = MODE_BISECT;
    e->seeds = nullptr;
    e->out20 = out20;
    e->job_nodes = nullptr;
    e->next = &next;
    e->tt = tts[i].data();
    sh->tts.push_back(tts[i].data());
    e->mask = (1u << tt_log2) - 1;
    memset(&e->st, 0, sizeof(e->st));
    e->sh = sh;
    e->lane_id = i;
    e->min_nodes = 0;  // donate from any job (the GPU waits for DONATE_MIN_NODES)
    envs[i] = e;
    memset(&L[i], 0, sizeof(Lane));
    L[i].stage = ST_TAKE;
    L[i].task = -1;
    L[i].owner = -1;
  }
  sh->eager = eager != 0;
  sh->cheap_limit = cheap_limit;
  uint64_t iters = 0;
  for (;;) {
    int live = 0;
    for (int i = 0; i < lanes; i++) live += L[i].stage != ST_IDLE;
    if (!live) break;
    if (++iters > 4000000000ull) return -2;
    sh->budget = lanes;
    int busy = 0;
    for (int i = 0; i < lanes; i++) busy += L[i].stage != ST_HUNGRY && L[i].stage != ST_IDLE;
    if (busy < free_below) {  // the kernel's free-running round, lane by lane
      const bool all_done = sh->pool.exhausted && sh->pool.busy == 0;
      for (int i = 0; i < lanes; i++) {
        if (L[i].stage == ST_HUNGRY && all_done) {
          sh->pool.hungry--;
          L[i].stage = ST_IDLE;
          continue;
        }
        if (task_abandoned(L[i], &sh->pool)) abort_task(L[i], *envs[i]);
        advance_free(L[i], *envs[i], free_steps, L[i].stage == ST_HUNGRY);
      }
      continue;
    }
    for (int i = 0; i < lanes; i++) {  // CHEAP (with abandoned helpers)
      if (task_abandoned(L[i], &sh->pool)) abort_task(L[i], *envs[i]);
      if (cheap_stage(L[i].stage)) advance_cheap(L[i], *envs[i]);
    }
    for (int i = 0; i < lanes; i++)
      if (L[i].stage == ST_ENTER && L[i].p.nplayed == 0) step_enter(L[i], *envs[i]);
    for (int i = 0; i < lanes; i++)
      if (L[i].stage == ST_ENTER && L[i].p.nplayed != 0) step_enter(L[i], *envs[i]);
    for (int ph = ST_MOVES_LEAD; ph <= ST_MOVES_FOLLOW; ph++)
      for (int i = 0; i < lanes; i++)
        if (L[i].stage == ph) {
          step_moves(L[i], *envs[i]);
          step_next(L[i], *envs[i]);
        }
  }
  for (int k = 0; k < MAX_TASKS; k++)
    if (sh->pool.state[k] != TASK_FREE) return -3;  // every task must be back in the pool
  if (sh->pool.busy || sh->pool.hungry || sh->pool.queued) return -4;  // and every count at zero
  for (int u : sh->users)
    if (u) return -5;  // every helper let go of its donor's TT
  if (stats) {
    memset(stats, 0, 14 * sizeof(uint64_t));
    for (auto* e : envs) {
      stats[0] += e->st.nodes;
      stats[1] += e->st.tt.probes;
      stats[2] += e->st.tt.hits;
      stats[3] += e->st.tt.stores;
      stats[4] += e->st.tt.bytes;
    }
    stats[12] = (uint64_t)sh->pool.posted;
    stats[13] = iters;
  }
  for (auto* e : envs) delete e;
  delete sh;
  return 0;
}


// n deals, jpd 5 or 20 jobs per deal, mode 0 (binary search) / 1 (stepping from seeds).
// stats[0..4] = nodes, probes, hits, stores, TT bytes; stats[5..11] = enter exits;
// stats[12] = accesses a bounds-checked build found out of range.
int replay_solve_hinted(const uint64_t* hands, long long n, int tt_log2, int jpd, int mode, const int8_t* seeds,
                        const int8_t* hints, int threads, int* out20, uint64_t* job_nodes, uint64_t* stats);
int replay_solve(const uint64_t* hands, long long n, int tt_log2, int jpd, int mode,
                 const int8_t* seeds, int threads, int* out20, uint64_t* job_nodes,
                 uint64_t* stats) {
  return replay_solve_hinted(hands, n, tt_log2, jpd, mode, seeds, nullptr, threads, out20, job_nodes, stats);
}

// replay_solve with the learned guide's root leads (hints: n*20, strain*4 + declarer; -1 =
// none), as ddg_solve_device_ex's d_hint20.
int replay_solve_hinted(const uint64_t* hands, long long n, int tt_log2, int jpd, int mode, const int8_t* seeds,
                        const int8_t* hints, int threads, int* out20, uint64_t* job_nodes, uint64_t* stats) {
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
      env->hints = hints;
      env->out20 = out20;
      env->job_nodes = job_nodes;
      env->next = &next;
      env->tt = tt.data();
      env->mask = (1u << tt_log2) - 1;
      memset(&env->st, 0, sizeof(env->st));
      Lane L;
      memset(&L, 0, sizeof(L));
      L.stage = ST_TAKE;
      L.owner = -1;
      while (L.stage != ST_IDLE) lane_step(L, *env);
      lane_stats[t] = env->st;
      delete env;
    });
  for (auto& th : pool) th.join();
  if (stats) {
    memset(stats, 0, 13 * sizeof(uint64_t));
    for (auto& s : lane_stats) {
      stats[12] += s.bounds;
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
