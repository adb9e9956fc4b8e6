// The batch kernel: a persistent block-phase machine over an atomic job queue.
//
// Each thread owns a solver lane (its own TT slice and frame stack in HBM); jobs (one
// (deal, strain), or one (deal, strain, declarer)) come from a global counter as lanes
// free up, so lanes that drew easy jobs keep working. The lanes' search state lives in
// shared memory, so any thread of the block can advance any lane. Each iteration of the
// block runs five phases in turn; a phase gathers the lanes that need it (one ballot per
// warp, then a block-wide select) and hands them to the first threads of the block:
//   CHEAP   returns, next moves, job starts (short, run back to back per lane)
//   LEAD    ENTER at a trick start: TT probe, QuickTricks, LaterTricks
//   FOLLOW  ENTER inside a trick: second-hand QuickTricks
//   MOVES   lead / follow move generation with the DDS weights, then the first move
// so warps run full and the whole block runs one code region at a time, instead of each
// warp's 32 lanes scattering over the stages and branches of the search.
#pragma once
#include "ddg_search.cuh"

namespace ddg {

// Device statistics block (u64 words).
enum {
  CNT_NEXT_JOB = 0,
  CNT_NODES = 1,
  CNT_PROBES = 2,
  CNT_HITS = 3,
  CNT_STORES = 4,
  CNT_TT_BYTES = 5,
  CNT_EXIT = 6,           // 7 words
  CNT_PHASE_WARPS = 13,   // 8 words: warp passes per phase
  CNT_PHASE_ITEMS = 21,   // 8 words: lanes served per phase
  CNT_JOBS_DONE = 29,
  CNT_ITERS = 30,         // block iterations
  CNT_TASKS = 31,         // tasks donated to helpers
  CNT_PHASE_CYCLES = 32,  // 8 words: SM cycles per phase, summed over blocks
  CNT_FAULTS = 38,        // blocks whose bounded queue wait gave up (never expected)
  CNT_BLOCKS_DONE = 39,   // blocks that ended with every lane idle (the solve is complete)
  CNT_BOUNDS = 40,        // bounds-checked builds: out-of-range accesses skipped (never expected)
  CNT_ENTRY_READS = 41,   // TT entries read by probes
  CNT_WORDS = 42
};

struct BatchArgs {
  const u64* hands;      // n * 4
  long long n_jobs;      // n * jpd
  int jpd;               // 5 or 20
  int mode;              // MODE_BISECT, or MODE_STEP with seeds
  const int8_t* seeds;   // n * 20 NS seeds, or null
  uint8_t* out20;        // n * 20
  u64* job_nodes;        // n * jpd, or null
  unsigned long long* counters;  // CNT_WORDS
  TTBucket* tt;          // lanes << tt_log2 buckets
  Frame* stacks;         // lanes * STACK_DEPTH
  u32* lane_gen;         // TT generation of each lane
  int tt_log2;
  int schedule;
  volatile int* stop;    // host-set stop flag (mapped memory), or null
  u64* job_end_ns;       // n * jpd completion times (device global timer, ns), or null
  u64* job_start_ns;     // n * jpd times the jobs were taken by a lane, or null
  TaskPool* tasks;       // helping: idle lanes take donated moves (tricks exact), or null
  int share_tt;          // helping: a helper searches in its donor's TT (else in its own)
  int* tt_users;         // helping with shared TTs: per lane, helpers searching in its TT
  int free_below;        // fewer busy lanes than this in a block: free-running rounds, no phases
  int free_steps;        // stages a lane runs per free-running round
  struct LaneSave* save; // resumable solve: lane states kept between launches, or null
  int resume;            // 1: lanes start from `save` (a later slice of the same solve)
  u64 slice_ns;          // resumable solve: each block stops this long after it starts (0 = never)
  unsigned long long* next_job;  // job queue head (counters + CNT_NEXT_JOB, or the stream's)
  // Stream mode (ring != null): deals come from a device ring the host keeps filling.
  const u64* ring;                         // slots * 4 hands; deal seq lives in slot seq & ring_mask
  const unsigned long long* published;     // deals published so far (device word, host-written)
  const int* closing;                      // 1: no deal will be published any more
  int* deal_done;                          // per slot: jobs of the deal finished
  struct CompRec* comp;                    // completion records (mapped host memory), slots of them
  unsigned long long* comp_tail;           // completion records written so far
  long long ring_mask;
  u64 idle_ns;                             // a block whose lanes found no deal this long ends
  int spread;            // phases hand their lanes round-robin over the block's warps
  int cheap_limit;       // most cheap stages a lane runs per pass (0 = until it needs more)
  long long rr_jobs;     // jobs 0..rr_jobs-1 are dealt to the lanes round-robin over the blocks
  int fuse_follow;       // ENTER inside a trick runs in the cheap pass (no FOLLOW phase)
  const int8_t* hint20;  // n * 20 root leads to try first (learned guide), -1 = none; or null
  int8_t* best20;        // n * 20 best leads found (the cutting root card), -1 = none; or null
  // One-job solves (ddg_solve_strain, ddg_ns_tricks): with `one_job` set, job 0 is strain
  // `one_strain` of deal 0, for declarer `one_decl` alone (-1 = all four). A zeroed
  // BatchArgs has it off. `first_target` is the binary search's first target (0 = 7).
  int one_job, one_strain, one_decl, first_target;
  int flat_moves;        // the lead-move phase spreads (lane, candidate) pairs over the block
  int free_pack;         // free-running rounds: busy lanes per warp; 0 = 1 up to 8 busy lanes, else 32
};

// One finished deal of a stream: its sequence number and table; `flag` = record index + 1,
// written last, tells the host the record is complete.
struct CompRec {
  unsigned long long seq;
  uint8_t tricks[20];
  unsigned flag;
};
static_assert(sizeof(CompRec) == 32, "completion record is 32 bytes");

__device__ __forceinline__ u64 global_ns() {
  u64 t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

struct LaneCounters {
  LaneStats s;
  u64 start_nodes;
  u64 tt_key;  // (deal, strain) key of the helper tasks the lane's TT holds, 0 = none
  u32 jobs_done;
};

// A lane between two slices of a resumable solve (HBM): its whole search state, the nodes
// its current job or task has taken so far, and its TT key.
struct LaneSave {
  Lane L;
  u64 progress;
  u64 tt_key;
};

// Start of a launch: a fresh lane, or the lane as the previous slice left it.
__device__ __forceinline__ void lane_begin(const BatchArgs& a, long long lane, Lane& L, LaneCounters& c) {
  memset(&c, 0, sizeof(LaneCounters));
  if (a.resume) {
    const LaneSave& sv = a.save[lane];
    L = sv.L;
    c.start_nodes = 0ull - sv.progress;  // work_nodes() = progress + this slice's nodes
    c.tt_key = sv.tt_key;
    return;
  }
  L.stage = ST_TAKE;
  L.job = -1;  // no job yet in this launch
  L.sp = 0;
  L.gen = a.lane_gen[lane];
  L.v = 0;
  L.r = 0;
  L.p.trick = 0;
  L.task = -1;
  L.owner = -1;
}

// End of a launch: the TT generation, and for a resumable solve the lane's state.
__device__ __forceinline__ void lane_end(const BatchArgs& a, long long lane, const Lane& L, const LaneCounters& c) {
  a.lane_gen[lane] = L.gen;
  if (a.save) {
    LaneSave& sv = a.save[lane];
    sv.L = L;
    sv.progress = c.s.nodes - c.start_nodes;
    sv.tt_key = c.tt_key;
  }
}

// The block's stop test (thread 0): the host's flag, or the end of the slice.
__device__ __forceinline__ bool stop_requested(const BatchArgs& a, u64 t_end) {
  return (a.stop && *a.stop) || (t_end && global_ns() > t_end);
}

struct DevEnv {
  const BatchArgs* a;
  Frame* stack;
  TTBucket* tt;
  u32 mask;
  LaneCounters* c;
  TaskPool* tp;           // null when helping is off
  const int* help_hint;   // block flag: hungry lanes outnumber queued tasks (this iteration)
  int* take_budget;       // stream: deals this block may still start this iteration
  long long lane;

  __device__ __forceinline__ LaneStats& stats() { return c->s; }
  __device__ __forceinline__ TaskPool* pool() { return tp; }
  __device__ __forceinline__ TTBucket* tt_of(int owner) const { return a->tt + ((long long)owner << a->tt_log2); }
  __device__ __forceinline__ long long self() const { return lane; }
  __device__ __forceinline__ bool share_tt() const { return a->share_tt != 0; }
  __device__ __forceinline__ void tt_users_add(int owner, int d) { atomicAdd(a->tt_users + owner, d); }
  __device__ __forceinline__ int tt_users(int owner) {
    __threadfence();  // the job's last task operations before the count is read
    return atom_load(a->tt_users + owner);
  }
  __device__ __forceinline__ bool want_donation() {
    if (!*help_hint) return false;
    const int q = atomicAdd(&tp->queued, 1);
    if (q < atom_load(&tp->hungry)) return true;
    atomicAdd(&tp->queued, -1);
    return false;
  }
  __device__ __forceinline__ void unreserve() { atomicAdd(&tp->queued, -1); }
  __device__ __forceinline__ int claim_start() { return (int)((lane * 61) + (global_ns() >> 12)); }
  __device__ __forceinline__ u64 work_nodes() { return c->s.nodes - c->start_nodes; }
  __device__ __forceinline__ void task_started() { c->start_nodes = c->s.nodes; }
  __device__ __forceinline__ u64& tt_key() { return c->tt_key; }
  __device__ __forceinline__ int cheap_limit() const { return a->cheap_limit; }
  __device__ __forceinline__ bool fuse_follow() const { return a->fuse_follow != 0; }
  // 1: a job; 0: no job will come; -1 (stream): none published yet.
  __device__ __forceinline__ int take(Lane& L) {
    unsigned long long job;
    const u64* hands;
    if (a->ring) {
      // A block takes its share of the waiting jobs per iteration, so that a few deals in
      // flight spread over all SMs instead of filling the block that polled first.
      const bool closing = *reinterpret_cast<const volatile int*>(a->closing) != 0;
      if (closing && !stream_more()) return 0;  // nothing more will come
      if (atomicSub(take_budget, 1) <= 0) return -1;
      if (!stream_take(job)) return -1;
      L.job = (long long)job;
      L.deal = L.job / a->jpd;
      hands = a->ring + (L.deal & a->ring_mask) * 4;
    } else {
      // A lane's first job of the launch is dealt round-robin over the blocks (job j to
      // block j mod grid), so a batch with fewer jobs than lanes spreads over every SM
      // instead of filling the first blocks; later jobs come from the shared counter.
      const long long t = lane - (long long)blockIdx.x * blockDim.x;
      const long long rr = t * gridDim.x + blockIdx.x;
      if (L.job < 0 && rr < a->rr_jobs) job = (unsigned long long)rr;
      else job = atomicAdd(a->next_job, 1ull) + (unsigned long long)a->rr_jobs;
      if ((long long)job >= a->n_jobs) return 0;
      L.job = (long long)job;
      L.deal = L.job / a->jpd;
      hands = a->hands + L.deal * 4;
    }
    int sub = (int)(L.job - L.deal * a->jpd);
    const ulonglong2* h = reinterpret_cast<const ulonglong2*>(hands);
    ulonglong2 x = h[0], y = h[1];
    L.p.h[0] = x.x;
    L.p.h[1] = x.y;
    L.p.h[2] = y.x;
    L.p.h[3] = y.y;
    if (a->jpd == 5) {
      L.strain = sub;
      L.decl = 0;
      L.last_decl = 3;
    } else {
      L.strain = sub >> 2;
      L.decl = sub & 3;
      L.last_decl = L.decl;
    }
    if (a->one_job) {
      L.strain = a->one_strain;
      L.decl = a->one_decl >= 0 ? a->one_decl : 0;
      L.last_decl = a->one_decl >= 0 ? a->one_decl : 3;
    }
    L.mode = a->mode;
    c->start_nodes = c->s.nodes;
    if (a->job_start_ns) a->job_start_ns[L.job] = global_ns();
    return 1;
  }
  // Stream: claims the next published job, if any.
  __device__ __forceinline__ bool stream_take(unsigned long long& job) {
    const long long avail = (long long)*reinterpret_cast<const volatile unsigned long long*>(a->published) * a->jpd;
    unsigned long long j = *reinterpret_cast<volatile unsigned long long*>(a->next_job);
    for (int tries = 0; tries < 8; tries++) {
      if ((long long)j >= avail) return false;
      const unsigned long long prev = atomicCAS(a->next_job, j, j + 1);
      if (prev == j) {
        job = j;
        return true;
      }
      j = prev;
    }
    return false;
  }
  // Stream, after `closing` was seen: were deals published that no lane has taken yet?
  __device__ __forceinline__ bool stream_more() {
    __threadfence();
    const long long avail = (long long)*reinterpret_cast<const volatile unsigned long long*>(a->published) * a->jpd;
    return (long long)*reinterpret_cast<volatile unsigned long long*>(a->next_job) < avail;
  }
  __device__ __forceinline__ int seed(const Lane& L) {
    if (a->mode == MODE_STEP) return (int)a->seeds[out_row(L) * 20 + L.strain * 4 + L.decl];
    return a->first_target ? a->first_target : 7;
  }
  __device__ __forceinline__ long long out_row(const Lane& L) const {
    return a->ring ? (L.deal & a->ring_mask) : L.deal;
  }
  __device__ __forceinline__ int root_hint(const Lane& L) {
    return a->hint20 ? (int)a->hint20[out_row(L) * 20 + L.strain * 4 + L.decl] : -1;
  }
  __device__ __forceinline__ void root_best(const Lane& L, int card) {
    if (a->best20) a->best20[out_row(L) * 20 + L.strain * 4 + L.decl] = (int8_t)card;
  }
  __device__ __forceinline__ void answer(const Lane& L, int ns) {
    a->out20[out_row(L) * 20 + L.strain * 4 + L.decl] = (uint8_t)((L.decl & 1) == 0 ? ns : 13 - ns);
  }
  __device__ __forceinline__ void job_done(const Lane& L) {
    if (a->job_nodes) a->job_nodes[L.job] = c->s.nodes - c->start_nodes;
    if (a->job_end_ns) a->job_end_ns[L.job] = global_ns();
    c->jobs_done++;
    if (a->ring) stream_job_done(L);
  }
  // Stream: the lane that finishes a deal's last job writes its completion record.
  __device__ __noinline__ void stream_job_done(const Lane& L) {
    const long long slot = L.deal & a->ring_mask;
    __threadfence();  // this job's answers before the count
    if (atomicAdd(a->deal_done + slot, 1) != a->jpd - 1) return;
    __threadfence();  // every job's answers are visible now
    const volatile uint8_t* o = a->out20 + slot * 20;
    const unsigned long long idx = atomicAdd(a->comp_tail, 1ull);
    volatile CompRec* r = a->comp + (idx & (unsigned long long)a->ring_mask);
    r->seq = (unsigned long long)L.deal;
    for (int k = 0; k < 20; k++) r->tricks[k] = o[k];
    // The slot's count is reset before the flag lets the host free the slot: a job of the
    // next deal in this slot must not find the old count.
    a->deal_done[slot] = 0;
    __threadfence_system();  // the record and the reset before the flag
    r->flag = (unsigned)idx + 1u;
  }
};

enum { PH_CHEAP = 0, PH_LEAD = 1, PH_FOLLOW = 2, PH_MOVES_LEAD = 3, PH_MOVES_FOLLOW = 4, PH_COUNT = 5 };

template <int BLOCK>
struct BlockShared {
  Lane lane[BLOCK];
  LaneCounters cnt[BLOCK];
  BatchArgs args;
  unsigned mask[BLOCK / 32];
  unsigned mask2[BLOCK / 32];  // free-running rounds: lanes waiting for a job or a task
  // flattened lead-move phase (run_moves_lead_flat), per position of the phase's list
  u64 fl_cand[BLOCK], fl_all[BLOCK];
  uint16_t fl_item[BLOCK], fl_off[BLOCK];
  int8_t fl_hint[BLOCK];
  int fl_wsum[BLOCK / 32];
  int16_t fl_score[BLOCK * 13];
  unsigned long long ph_warps[PH_COUNT], ph_items[PH_COUNT], iters;
  int stop;
  int help_hint;    // hungry lanes outnumber queued tasks (read once per iteration)
  int take_budget;  // stream: jobs this block may still take this iteration
  int claim_slots;  // hungry lanes of this block that may look for a task this iteration
  int all_done;     // no job left anywhere and no lane busy: hungry lanes stop
  unsigned long long ph_cycles[PH_COUNT];
  unsigned long long free_rounds, free_cycles;  // free-running rounds and their SM cycles
  // Stage queues of the queue kernel: per phase a ring of lane ids + 1 (0 = slot not yet
  // written). Every lane is in at most one ring, so a ring never holds more than BLOCK.
  uint16_t q[PH_COUNT][BLOCK];
  unsigned qhead[PH_COUNT], qtail[PH_COUNT];
  unsigned parked[BLOCK / 32];  // lanes waiting on the task pool (HUNGRY, WAIT)
  int live;                     // lanes not IDLE
  int fault;                    // a queue slot was never written (bounded wait gave up)
  u64 idle_since;               // stream: global time since which no lane had work (0 = busy)
  int idle_exit;                // stream: waiting lanes end
};

// Position of the r-th (0-based) set bit of m (r < popc(m)).
__device__ __forceinline__ int select_bit(unsigned m, int r) {
  int pos = 0, c;
  c = __popc(m & 0xFFFFu);
  if (r >= c) { r -= c; m >>= 16; pos += 16; }
  c = __popc(m & 0xFFu);
  if (r >= c) { r -= c; m >>= 8; pos += 8; }
  c = __popc(m & 0xFu);
  if (r >= c) { r -= c; m >>= 4; pos += 4; }
  c = __popc(m & 0x3u);
  if (r >= c) { r -= c; m >>= 2; pos += 2; }
  return pos + (r >= (int)(m & 1u) ? 1 : 0);
}

template <int BLOCK>
__device__ __forceinline__ DevEnv lane_env(BlockShared<BLOCK>& sh, long long lane, int slot) {
  DevEnv env;
  env.a = &sh.args;
  env.tt = sh.args.tt + (lane << sh.args.tt_log2);
  env.mask = (1u << sh.args.tt_log2) - 1;
  env.stack = sh.args.stacks + lane * STACK_DEPTH;
  env.c = &sh.cnt[slot];
  env.tp = sh.args.tasks;
  env.help_hint = &sh.help_hint;
  env.take_budget = &sh.take_budget;
  env.lane = lane;
  return env;
}

// One phase: the lanes that need it go, in block order, to threads 0, 1, 2, ...
template <int BLOCK, int PH>
__device__ __forceinline__ void run_phase(BlockShared<BLOCK>& sh, long long base, int tid) {
  const int wid = tid >> 5, ln = tid & 31;
  const Lane& me = sh.lane[tid];
  bool want;
  if (PH == PH_CHEAP) {  // hungry lanes only when a task may be waiting (or to stop them)
    want = (cheap_stage(me.stage) && (me.stage != ST_HUNGRY || sh.claim_slots > 0 || sh.all_done)) ||
           (sh.args.tasks && task_abandoned(me, sh.args.tasks));
    if (sh.args.ring) {
      // Stream: of the lanes waiting for a job, only as many as the block may take this
      // iteration poll the ring; the others stay out of the pass instead of each reading
      // the published and taken counts in global memory.
      const bool waiting = me.stage == ST_TAKE;
      const unsigned mt = __ballot_sync(0xFFFFFFFFu, waiting);
      if (ln == 0) sh.mask2[wid] = mt;
      __syncthreads();
      if (waiting) {
        int rank = __popc(mt & ((1u << ln) - 1));
        for (int w = 0; w < wid; w++) rank += __popc(sh.mask2[w]);
        want = rank < sh.take_budget;
      }
    }
  } else if (PH == PH_LEAD) {
    want = me.stage == ST_ENTER && me.p.nplayed == 0;
  }
  else if (PH == PH_FOLLOW) want = me.stage == ST_ENTER && me.p.nplayed != 0;
  else if (PH == PH_MOVES_LEAD) want = me.stage == ST_MOVES_LEAD;
  else want = me.stage == ST_MOVES_FOLLOW;
  const unsigned m = __ballot_sync(0xFFFFFFFFu, want);
  if (ln == 0) sh.mask[wid] = m;
  __syncthreads();
  // Position of this thread in the phase's list: packed (thread t takes item t, so the
  // items fill whole warps) or spread (item p goes to lane p / warps of warp p % warps, so
  // every warp of the block takes a share and fewer lanes share each warp's divergence).
  const int pos = sh.args.spread ? (tid & 31) * (BLOCK / 32) + wid : tid;
  int total = 0, item = -1;
#pragma unroll
  for (int w = 0; w < BLOCK / 32; w++) {
    const unsigned mw = sh.mask[w];
    const int c = __popc(mw);
    if (item < 0 && pos < total + c) item = w * 32 + select_bit(mw, pos - total);
    total += c;
  }
  if (tid == 0 && total) {
    sh.ph_items[PH] += total;
    sh.ph_warps[PH] += (total + 31) >> 5;
  }
  if (item >= 0) {
    DevEnv env = lane_env(sh, base + item, item);
    Lane& L = sh.lane[item];
    if (PH == PH_CHEAP) {
      if (env.tp && task_abandoned(L, env.tp)) abort_task(L, env);
      if (L.stage == ST_HUNGRY) {
        if (sh.all_done) {
          atomicAdd(&env.tp->hungry, -1);
          L.stage = ST_IDLE;
        } else if (atomicSub(&sh.claim_slots, 1) <= 0) {
          L.stage = ST_HUNGRY;  // no claim this iteration
        } else {
          advance_cheap(L, env);
        }
      } else {
        advance_cheap(L, env);
      }
    } else if (PH == PH_LEAD || PH == PH_FOLLOW) {
      step_enter(L, env);
    } else {
      step_moves(L, env);
      step_next(L, env);  // a fresh node plays its first candidate (never a skipped one)
    }
  }
  __syncthreads();
}

// Stage class of a lane in a free-running round: 0 the cheap stages (returns, next moves,
// job starts, waits), 1 ENTER at a trick start, 2 ENTER inside a trick, 3 lead moves, 4
// follow moves; -1 idle.
__device__ __forceinline__ int free_class(const Lane& L) {
  switch (L.stage) {
    case ST_ENTER: return L.p.nplayed == 0 ? 1 : 2;
    case ST_MOVES_LEAD: return 3;
    case ST_MOVES_FOLLOW: return 4;
    case ST_IDLE: return -1;
    default: return 0;
  }
}

// The lead-move phase with its work flattened: every (lane, candidate) pair of the phase
// is one item, and the items are spread over all threads of the block, so the DDS lead
// weights of one lane's candidates are computed side by side instead of in a loop whose
// length differs from lane to lane of a warp. Each lane's thread then orders its
// candidates exactly as gen_moves_lead does (arrival order highest card first, stable by
// weight), so the search and its node counts are unchanged.
template <int BLOCK>
__device__ __forceinline__ void run_moves_lead_flat(BlockShared<BLOCK>& sh, long long base, int tid) {
  const int wid = tid >> 5, ln = tid & 31;
  const bool want = sh.lane[tid].stage == ST_MOVES_LEAD;
  const unsigned m = __ballot_sync(0xFFFFFFFFu, want);
  if (ln == 0) sh.mask[wid] = m;
  __syncthreads();
  int total = 0, item = -1;
#pragma unroll
  for (int w = 0; w < BLOCK / 32; w++) {
    const unsigned mw = sh.mask[w];
    const int c = __popc(mw);
    if (item < 0 && tid < total + c) item = w * 32 + select_bit(mw, tid - total);
    total += c;
  }
  // 1. each item's candidates (and the root hint, as step_moves takes it)
  int cnt = 0;
  u64 cand = 0;
  DevEnv env;
  if (item >= 0) {
    env = lane_env(sh, base + item, item);
    const Lane& L = sh.lane[item];
    int hint = frame_hint(L.f);
    if (hint < 0 && L.sp == 0 && L.task < 0) {
      const int h = env.root_hint(L);
      if (h >= 0 && h < 64 && (hand_at(L.p.h, L.p.leader) >> h & 1)) hint = h;
    }
    u64 all;
    cand = candidates(L.p, L.p.leader, all);
    cnt = popc(cand);
    sh.fl_cand[tid] = cand;
    sh.fl_all[tid] = all;
    sh.fl_item[tid] = (uint16_t)item;
    sh.fl_hint[tid] = (int8_t)hint;
  }
  // 2. where each item's candidates start in the flat list (exclusive prefix sum)
  int incl = cnt;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int v = __shfl_up_sync(0xFFFFFFFFu, incl, d);
    if (ln >= d) incl += v;
  }
  if (ln == 31) sh.fl_wsum[wid] = incl;
  __syncthreads();
  int off = incl - cnt, work = 0;
#pragma unroll
  for (int w = 0; w < BLOCK / 32; w++) {
    if (w < wid) off += sh.fl_wsum[w];
    work += sh.fl_wsum[w];
  }
  if (item >= 0) sh.fl_off[tid] = (uint16_t)off;
  __syncthreads();
  // 3. the weights, one (lane, candidate) pair per thread at a time
  for (int w = tid; w < work; w += BLOCK) {
    int lo = 0, hi = total - 1;  // the last item whose candidates start at or before w
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (sh.fl_off[mid] <= w) lo = mid;
      else hi = mid - 1;
    }
    u64 rest = sh.fl_cand[lo];
    for (int k = w - sh.fl_off[lo]; k > 0; k--) rest ^= card_bit(top_bit(rest));
    const int card = top_bit(rest);
    const Lane& L = sh.lane[sh.fl_item[lo]];
    Hands hs;
    for (int i = 0; i < 4; i++) hs.h[i] = L.p.h[i];
    const int hint = sh.fl_hint[lo];
    const bool hinted = hint >= 0 && alike(hand_at(L.p.h, L.p.leader), sh.fl_all[lo], hint, card);
    sh.fl_score[w] = (int16_t)lead_weight(hs, L.top, L.p.trump, L.p.left, L.p.leader, card, hinted);
  }
  __syncthreads();
  // 4. each lane's candidates ordered as gen_moves_lead orders them, then its first move
  if (item >= 0) {
    Lane& L = sh.lane[item];
    int n = 0, score[13], card_of[13];
    u64 rest = cand;
    for (int k = 0; k < cnt; k++) {
      const int card = top_bit(rest);
      rest ^= card_bit(card);
      insert_move(score, card_of, n, card, sh.fl_score[off + k]);
    }
    pack_moves(L.f, card_of, n);
    L.stage = ST_NEXT;
    step_next(L, env);
  }
  if (tid == 0 && total) {
    sh.ph_items[PH_MOVES_LEAD] += total;
    sh.ph_warps[PH_MOVES_LEAD] += (total + 31) >> 5;
  }
  __syncthreads();
}

template <int BLOCK>
__device__ __forceinline__ void block_counters(BlockShared<BLOCK>& sh, const BatchArgs& a, int tid);

// BLOCK threads (= lanes) per block; MINB resident blocks per SM asked of the register
// allocator.
template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) batch_kernel(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BlockShared<BLOCK>& sh = *reinterpret_cast<BlockShared<BLOCK>*>(smem_raw);
  const int tid = threadIdx.x;
  const long long base = (long long)blockIdx.x * BLOCK;
  lane_begin(a, base + tid, sh.lane[tid], sh.cnt[tid]);
  const u64 t_end = a.slice_ns ? global_ns() + a.slice_ns : 0;
  if (tid < PH_COUNT) {
    sh.ph_warps[tid] = 0;
    sh.ph_items[tid] = 0;
    sh.ph_cycles[tid] = 0;
  }
  if (tid == 0) {
    sh.args = a;
    sh.stop = 0;
    sh.iters = 0;
    sh.help_hint = 0;
    sh.claim_slots = 0;
    sh.all_done = 0;
    sh.free_rounds = 0;
    sh.free_cycles = 0;
    sh.idle_since = 0;
    sh.idle_exit = 0;
  }
  __syncthreads();
  for (unsigned iter = 0;; iter++) {
    if (tid == 0 && (iter & 15u) == 15u && stop_requested(a, t_end)) sh.stop = 1;
    if (!__syncthreads_or(sh.lane[tid].stage != ST_IDLE)) break;
    if (sh.stop) {
      if (a.save) break;  // resumable: the lanes are kept for the next slice
      sh.lane[tid].stage = ST_IDLE;  // host time limit: unfinished results stay 255
      continue;
    }
    if (tid == 0) {
      sh.iters++;
      if (a.ring) {  // this block's share of the jobs waiting in the ring
        const long long waiting =
            (long long)*reinterpret_cast<const volatile unsigned long long*>(a.published) * a.jpd -
            (long long)*reinterpret_cast<const volatile unsigned long long*>(a.next_job);
        sh.take_budget = (int)((waiting > 0 ? waiting : 0) / gridDim.x) + 1;
      }
      if (a.tasks) {  // one read of the helping counters per block and iteration
        const int q = atom_load(&a.tasks->queued), h = atom_load(&a.tasks->hungry);
        sh.help_hint = h > q;
        sh.claim_slots = q > 32 ? 32 : q;
        sh.all_done = atom_load(&a.tasks->exhausted) && atom_load(&a.tasks->busy) == 0;
      }
    }
    int st0 = sh.lane[tid].stage;
    int busy_here = __syncthreads_count(st0 != ST_HUNGRY && st0 != ST_IDLE);
    if (a.ring) {
      // Stream: lanes waiting for a deal (TAKE) are not work. A block with nothing to do
      // naps between polls of the ring, and after idle_ns without work its waiting lanes
      // end (the host launches the kernel again when it publishes more).
      busy_here = __syncthreads_count(st0 != ST_HUNGRY && st0 != ST_IDLE && st0 != ST_TAKE);
      if (busy_here == 0) {
        if (tid == 0) {
          const u64 now = global_ns();
          if (!sh.idle_since) sh.idle_since = now;
          else if (now - sh.idle_since > a.idle_ns) sh.idle_exit = 1;
        }
        __nanosleep(20000);
      } else if (tid == 0) {
        sh.idle_since = 0;
      }
      __syncthreads();
      if (sh.idle_exit && st0 == ST_TAKE) sh.lane[tid].stage = ST_IDLE;
    }
    if (busy_here < a.free_below) {
      // Few busy lanes: each lane runs on a thread of its own for a while, no phases. The
      // lanes with search work go first, round-robin over the round's nw warps (the k-th
      // to warp k mod nw, the (k div nw)-th thread of it); lanes waiting for a job or a
      // task come after them.
      const long long f0 = clock64();
      {
        const int wid = tid >> 5, ln = tid & 31;
        const int stg = sh.lane[tid].stage;
        const bool work = stg != ST_IDLE && stg != ST_TAKE && stg != ST_HUNGRY;
        const unsigned mw = __ballot_sync(0xFFFFFFFFu, work);
        const unsigned mo = __ballot_sync(0xFFFFFFFFu, stg == ST_TAKE || stg == ST_HUNGRY);
        if (ln == 0) {
          sh.mask[wid] = mw;
          sh.mask2[wid] = mo;
        }
      }
      __syncthreads();
      // The busy lanes go to the first nw warps, nw = ceil(busy / pack) (at most all of
      // them), the waiting lanes to the other threads. Few warps share their instruction fetches
      // (spread over all 16 warps, 68 busy lanes per block stalled 4.6 cycles per issue
      // on instruction fetch and searched 74 M nodes/s over the GPU; packed 32 to a warp,
      // 169 M); a handful of lanes runs faster one to a warp, on the SM's four
      // schedulers (5 busy lanes per block: 36.8 M against 32.2 M packed). pack =
      // free_pack, or by default 1 up to 8 busy lanes and 32 above.
      int nwork = 0;
#pragma unroll
      for (int w = 0; w < BLOCK / 32; w++) nwork += __popc(sh.mask[w]);
      const int pack = a.free_pack > 0 && a.free_pack <= 32 ? a.free_pack : (nwork <= 8 ? 1 : 32);
      int nw = (nwork + pack - 1) / pack;
      if (nw > BLOCK / 32) nw = BLOCK / 32;
      if (nw < 1) nw = 1;
      // Thread (warp w < nw, lane l) takes busy lane number l*nw + w when that is below
      // nwork; the other threads, those of warps nw.. first, then the unused ones of the
      // first nw warps, take the waiting lanes in order (BLOCK threads hold all BLOCK lanes).
      const int wid = tid >> 5, p = (tid & 31) * nw + wid;
      const bool takes_work = wid < nw && p < nwork;
      const int rank = takes_work ? p : wid >= nw ? tid - nw * 32 : (BLOCK - nw * 32) + (p - nwork);
      int item = -1, total = 0;
#pragma unroll
      for (int w = 0; w < BLOCK / 32; w++) {
        const unsigned mw = takes_work ? sh.mask[w] : sh.mask2[w];
        const int c = __popc(mw);
        if (item < 0 && rank < total + c) item = w * 32 + select_bit(mw, rank - total);
        total += c;
      }
      // Each warp then steps its lanes, one stage at a time, choosing each time the stage
      // class that most of its lanes are in (the warp-synchronous stage machine of the
      // reference's wave_kernel, gpu/gpu_main.cu:61-152, per warp): the lanes of one step
      // run one code region together instead of each thread walking its own lane through
      // every stage, which would scatter a warp over the whole kernel's code. A lane that
      // can make no progress (waiting for a job, a task or a helper) sits out the round.
      DevEnv env;
      bool parked = true, may_claim = false;
      if (item >= 0) {
        Lane& L = sh.lane[item];
        if (L.stage == ST_HUNGRY && sh.all_done) {
          atomicAdd(&a.tasks->hungry, -1);
          L.stage = ST_IDLE;
        } else if (L.stage != ST_IDLE) {
          env = lane_env(sh, base + item, item);
          if (env.tp && task_abandoned(L, env.tp)) abort_task(L, env);
          may_claim = L.stage == ST_HUNGRY && atomicSub(&sh.claim_slots, 1) > 0;
          parked = false;
        }
      }
      for (int k = 0; k < a.free_steps; k++) {
        const int cls = parked ? -1 : free_class(sh.lane[item]);
        int best = -1, best_n = 0;
#pragma unroll
        for (int c = 0; c < 5; c++) {
          const int cnt = __popc(__ballot_sync(0xFFFFFFFFu, cls == c));
          if (cnt > best_n) {
            best_n = cnt;
            best = c;
          }
        }
        if (best < 0) break;  // every lane of the warp is idle or waiting
        if (cls == best) {
          Lane& L = sh.lane[item];
          const int before = L.stage;
          advance_free(L, env, 1, may_claim && before == ST_HUNGRY);
          if (before == ST_HUNGRY && L.stage != ST_HUNGRY) may_claim = false;
          if (L.stage == ST_IDLE ||
              ((before == ST_TAKE || before == ST_HUNGRY || before == ST_WAIT) && L.stage == before))
            parked = true;
        }
        __syncwarp();
      }
      __syncthreads();
      if (tid == 0) {
        sh.free_rounds++;
        sh.free_cycles += clock64() - f0;
      }
      continue;
    }
    long long t0 = clock64();
    run_phase<BLOCK, PH_CHEAP>(sh, base, tid);
    long long t1 = clock64();
    run_phase<BLOCK, PH_LEAD>(sh, base, tid);
    long long t2 = clock64();
    run_phase<BLOCK, PH_FOLLOW>(sh, base, tid);
    long long t3 = clock64();
    if (sh.args.flat_moves) run_moves_lead_flat<BLOCK>(sh, base, tid);
    else run_phase<BLOCK, PH_MOVES_LEAD>(sh, base, tid);
    long long t4 = clock64();
    run_phase<BLOCK, PH_MOVES_FOLLOW>(sh, base, tid);
    if (tid == 0) {
      long long t5 = clock64();
      sh.ph_cycles[PH_CHEAP] += t1 - t0;
      sh.ph_cycles[PH_LEAD] += t2 - t1;
      sh.ph_cycles[PH_FOLLOW] += t3 - t2;
      sh.ph_cycles[PH_MOVES_LEAD] += t4 - t3;
      sh.ph_cycles[PH_MOVES_FOLLOW] += t5 - t4;
    }
  }
  lane_end(a, base + tid, sh.lane[tid], sh.cnt[tid]);
  const int busy_left = __syncthreads_or(sh.lane[tid].stage != ST_IDLE);
  if (tid == 0 && !busy_left) atomicAdd(a.counters + CNT_BLOCKS_DONE, 1ull);
  block_counters(sh, a, tid);
}

// Phase queue of a lane's next stage, or -1 (parked on the task pool) / -2 (idle).
__device__ __forceinline__ int next_queue(const Lane& L) {
  switch (L.stage) {
    case ST_ENTER: return L.p.nplayed == 0 ? PH_LEAD : PH_FOLLOW;
    case ST_MOVES_LEAD: return PH_MOVES_LEAD;
    case ST_MOVES_FOLLOW: return PH_MOVES_FOLLOW;
    case ST_HUNGRY:
    case ST_WAIT: return -1;
    case ST_IDLE: return -2;
    default: return PH_CHEAP;
  }
}

// Hands lane `lane` (held by this thread) to the queue of its next stage. All threads of
// the warp call this; `active` says whether this thread holds a lane.
template <int BLOCK>
__device__ __forceinline__ void route_lane(BlockShared<BLOCK>& sh, bool active, int lane, int ln) {
  const int nq = active ? next_queue(sh.lane[lane]) : -3;
  __threadfence_block();  // the lane's state is written before another warp can take it
  const unsigned peers = __match_any_sync(0xFFFFFFFFu, nq);
  if (nq >= 0) {
    const int leader = __ffs(peers) - 1;
    const int rank = __popc(peers & ((1u << ln) - 1));
    unsigned slot = 0;
    if (ln == leader) slot = atomicAdd(&sh.qtail[nq], (unsigned)__popc(peers));
    slot = __shfl_sync(peers, slot, leader) + rank;
    reinterpret_cast<volatile uint16_t*>(sh.q[nq])[slot % BLOCK] = (uint16_t)(lane + 1);
  } else if (nq == -1) {
    atomicOr(&sh.parked[lane >> 5], 1u << (lane & 31));
  } else if (nq == -2) {
    if (ln == __ffs(peers) - 1) atomicSub(&sh.live, __popc(peers));
  }
}

// The queue kernel: the same stages and phases as batch_kernel, without block barriers.
// Each warp loops on its own: it takes up to 32 lanes from the fullest phase queue of its
// block, runs that phase for them and hands each lane to the queue of its next stage.
// Warps never wait for each other (no __syncthreads in the loop), a lane's next stage can
// run as soon as any warp is free, and a phase with few lanes costs only those lanes.
template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) queue_kernel(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BlockShared<BLOCK>& sh = *reinterpret_cast<BlockShared<BLOCK>*>(smem_raw);
  const int tid = threadIdx.x, ln = tid & 31;
  const long long base = (long long)blockIdx.x * BLOCK;
  lane_begin(a, base + tid, sh.lane[tid], sh.cnt[tid]);
  const u64 t_end = a.slice_ns ? global_ns() + a.slice_ns : 0;
  for (int p = 0; p < PH_COUNT; p++) sh.q[p][tid] = 0;
  if (tid < PH_COUNT) {
    sh.ph_warps[tid] = 0;
    sh.ph_items[tid] = 0;
    sh.ph_cycles[tid] = 0;
    sh.qhead[tid] = 0;
    sh.qtail[tid] = 0;
  }
  if (tid < BLOCK / 32) sh.parked[tid] = 0;
  if (tid == 0) {
    sh.args = a;
    sh.stop = 0;
    sh.iters = 0;
    sh.help_hint = 0;
    sh.claim_slots = 0;
    sh.all_done = 0;
    sh.free_rounds = 0;
    sh.free_cycles = 0;
    sh.live = 0;
    sh.fault = 0;
  }
  __syncthreads();
  route_lane(sh, sh.lane[tid].stage != ST_IDLE, tid, ln);  // every lane to its first queue
  if (sh.lane[tid].stage != ST_IDLE) atomicAdd(&sh.live, 1);
  __syncthreads();
  volatile unsigned* vhead = sh.qhead;
  volatile unsigned* vtail = sh.qtail;
  volatile int* vlive = &sh.live;
  volatile int* vstop = &sh.stop;
  volatile int* vfault = &sh.fault;
  unsigned poll_word = (unsigned)(tid >> 5);
  for (unsigned loop = 0;; loop++) {
    if (__shfl_sync(0xFFFFFFFFu, (*vstop | *vfault), 0)) break;  // warp-uniform
    if (ln == 0 && (loop & 63u) == 63u && stop_requested(a, t_end)) sh.stop = 1;
    if (a.tasks && ln == 0 && (loop & 15u) == 0) {
      const int q = atom_load(&a.tasks->queued), h = atom_load(&a.tasks->hungry);
      sh.help_hint = h > q;
      sh.all_done = atom_load(&a.tasks->exhausted) && atom_load(&a.tasks->busy) == 0;
    }
    // Lane 0 picks the fullest queue and claims up to 32 of its lanes.
    int ph = -1;
    unsigned h0 = 0, n = 0;
    if (ln == 0) {
      unsigned best = 0;
      for (int p = 0; p < PH_COUNT; p++) {
        const unsigned hd = vhead[p];  // head first: it never passes the tail read after it
        const unsigned b = vtail[p] - hd;
        if (b > best) {
          best = b;
          ph = p;
        }
      }
      if (ph >= 0) {
        h0 = vhead[ph];
        const unsigned avail = vtail[ph] - h0;
        n = avail < 32u ? avail : 32u;
        if (n == 0 || atomicCAS(&sh.qhead[ph], h0, h0 + n) != h0) ph = -2;  // lost the race: retry
      }
    }
    ph = __shfl_sync(0xFFFFFFFFu, ph, 0);
    if (ph == -2) continue;
    const bool poll = ph < 0 || (loop & 7u) == 7u;
    if (ph >= 0) {
      h0 = __shfl_sync(0xFFFFFFFFu, h0, 0);
      n = __shfl_sync(0xFFFFFFFFu, n, 0);
      int lane = -1;
      if ((unsigned)ln < n) {
        volatile uint16_t* slot = reinterpret_cast<volatile uint16_t*>(sh.q[ph]) + ((h0 + ln) % BLOCK);
        unsigned v = 0;
        for (int k = 0; k < (1 << 20) && (v = *slot) == 0; k++) {
        }
        if (v == 0) {
          *vfault = 1;  // the producer never wrote the slot: give up on the whole block
        } else {
          *slot = 0;
          lane = (int)v - 1;
        }
        __threadfence_block();  // read the lane's state only after taking it
      }
      const long long t0 = clock64();
      if (lane >= 0) {
        DevEnv env = lane_env(sh, base + lane, lane);
        Lane& L = sh.lane[lane];
        if (ph == PH_CHEAP) {
          if (env.tp && task_abandoned(L, env.tp)) abort_task(L, env);
          advance_cheap(L, env);
        } else if (ph == PH_LEAD || ph == PH_FOLLOW) {
          step_enter(L, env);
        } else {
          step_moves(L, env);
          step_next(L, env);
        }
      }
      route_lane(sh, lane >= 0, lane, ln);
      if (ln == 0) {
        atomicAdd(&sh.ph_items[ph], (unsigned long long)n);
        atomicAdd(&sh.ph_warps[ph], 1ull);
        atomicAdd(&sh.ph_cycles[ph], (unsigned long long)(clock64() - t0));
        atomicAdd(&sh.iters, 1ull);
      }
    }
    if (poll) {
      // Lanes parked on the task pool: one word of the block at a time.
      poll_word = (poll_word + 1) % (BLOCK / 32);
      unsigned m = 0;
      if (ln == 0 && reinterpret_cast<volatile unsigned*>(sh.parked)[poll_word])
        m = atomicExch(&sh.parked[poll_word], 0u);
      m = __shfl_sync(0xFFFFFFFFu, m, 0);
      __threadfence_block();
      int lane = -1;
      if (m) {
        const int c = __popc(m);
        if (ln < c) lane = (int)(poll_word * 32 + select_bit(m, ln));
        // Hungry lanes look for a task only as far as tasks are queued.
        const unsigned hm = __ballot_sync(0xFFFFFFFFu, lane >= 0 && sh.lane[lane].stage == ST_HUNGRY);
        int quota = 0;
        if (ln == 0 && hm) quota = atom_load(&a.tasks->queued);
        quota = __shfl_sync(0xFFFFFFFFu, quota, 0);
        if (lane >= 0) {
          DevEnv env = lane_env(sh, base + lane, lane);
          Lane& L = sh.lane[lane];
          if (env.tp && task_abandoned(L, env.tp)) abort_task(L, env);
          if (L.stage == ST_HUNGRY) {
            if (*reinterpret_cast<volatile int*>(&sh.all_done)) {
              atomicAdd(&env.tp->hungry, -1);
              L.stage = ST_IDLE;
            } else if (__popc(hm & ((1u << ln) - 1)) < quota) {
              advance_cheap(L, env);
            }
          } else {
            advance_cheap(L, env);
          }
        }
        route_lane(sh, lane >= 0, lane, ln);
      } else if (ph < 0) {
        if (__shfl_sync(0xFFFFFFFFu, *vlive, 0) == 0) break;
        __nanosleep(256);
      }
    }
  }
  __syncthreads();
  lane_end(a, base + tid, sh.lane[tid], sh.cnt[tid]);
  if (tid == 0 && sh.fault) atomicAdd(a.counters + CNT_FAULTS, 1ull);
  if (tid == 0 && sh.live == 0) atomicAdd(a.counters + CNT_BLOCKS_DONE, 1ull);
  __syncthreads();
  block_counters(sh, a, tid);
}

template <int BLOCK>
__device__ __forceinline__ void block_counters(BlockShared<BLOCK>& sh, const BatchArgs& a, int tid) {
  // Block sums of the counters, one atomic per word per block.
  if (tid < CNT_WORDS) {
    unsigned long long sum = 0;
    for (int t = 0; t < BLOCK; t++) {
      const LaneCounters& c = sh.cnt[t];
      switch (tid) {
        case CNT_NODES: sum += c.s.nodes; break;
        case CNT_PROBES: sum += c.s.tt.probes; break;
        case CNT_HITS: sum += c.s.tt.hits; break;
        case CNT_STORES: sum += c.s.tt.stores; break;
        case CNT_TT_BYTES: sum += c.s.tt.bytes; break;
        case CNT_JOBS_DONE: sum += c.jobs_done; break;
        case CNT_BOUNDS: sum += c.s.bounds; break;
        case CNT_ENTRY_READS: sum += c.s.tt.entry_reads; break;
        default:
#ifdef DDG_EXIT_COUNTS
          if (tid >= CNT_EXIT && tid < CNT_EXIT + 7) sum += c.s.enter_exit[tid - CNT_EXIT];
#endif
          break;
      }
    }
    if (tid >= CNT_PHASE_WARPS && tid < CNT_PHASE_WARPS + PH_COUNT) sum = sh.ph_warps[tid - CNT_PHASE_WARPS];
    if (tid >= CNT_PHASE_ITEMS && tid < CNT_PHASE_ITEMS + PH_COUNT) sum = sh.ph_items[tid - CNT_PHASE_ITEMS];
    if (tid == CNT_ITERS) sum = sh.iters;
    if (tid >= CNT_PHASE_CYCLES && tid < CNT_PHASE_CYCLES + PH_COUNT) sum = sh.ph_cycles[tid - CNT_PHASE_CYCLES];
    if (tid == CNT_PHASE_CYCLES + PH_COUNT) sum = sh.free_cycles;
    if (tid == CNT_PHASE_ITEMS + PH_COUNT) sum = sh.free_rounds;
    if (tid != CNT_NEXT_JOB && tid != CNT_FAULTS && tid != CNT_BLOCKS_DONE && sum) atomicAdd(a.counters + tid, sum);
  }
}

}  // namespace ddg
