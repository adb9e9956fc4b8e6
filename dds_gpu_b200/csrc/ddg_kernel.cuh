// The batch kernel: a persistent, warp-synchronous stage machine over an atomic job queue.
//
// Each thread is a solver lane with its own TT slice and frame stack in HBM; jobs
// (one (deal, strain), or one (deal, strain, declarer)) are taken from a global counter as
// lanes free up, so lanes that drew easy jobs keep working. In every warp iteration the
// warp picks one stage present among its lanes (a single __reduce_or_sync of the lanes'
// stage bits) and only the lanes in that stage run it: the cheap stages (RET, NEXT,
// ROOT, TAKE) go first, so lanes gather at ENTER, the expensive and most divergent stage,
// and run it together. Per-lane counters live in shared memory, not registers.
#pragma once
#include "ddg_search.cuh"

namespace ddg {

enum { STACK_DEPTH = 54 };  // frames per lane: at most 52 plies + the root

// Device statistics block (u64 words).
enum {
  CNT_NEXT_JOB = 0,
  CNT_NODES = 1,
  CNT_PROBES = 2,
  CNT_HITS = 3,
  CNT_STORES = 4,
  CNT_TT_BYTES = 5,
  CNT_EXIT = 6,          // 7 words
  CNT_STAGE_ITERS = 13,  // 6 words
  CNT_STAGE_LANES = 19,  // 6 words
  CNT_JOBS_DONE = 25,
  CNT_WORDS = 32
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
};

__device__ __forceinline__ u64 global_ns() {
  u64 t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

struct LaneCounters {
  LaneStats s;
  u64 start_nodes;
  u32 jobs_done;
};

// Dynamic shared memory of a block: lane states, counters, per-warp stage tallies.
template <int BLOCK>
struct BlockShared {
  Lane lane[BLOCK];
  LaneCounters cnt[BLOCK];
  unsigned long long stage[BLOCK / 32][12];
};

struct DevEnv {
  const BatchArgs* a;
  Frame* stack;
  TTBucket* tt;
  u32 mask;
  LaneCounters* c;

  __device__ __forceinline__ LaneStats& stats() { return c->s; }
  __device__ __forceinline__ bool take(Lane& L) {
    unsigned long long job = atomicAdd(a->counters + CNT_NEXT_JOB, 1ull);
    if ((long long)job >= a->n_jobs) return false;
    L.job = (long long)job;
    L.deal = L.job / a->jpd;
    int sub = (int)(L.job - L.deal * a->jpd);
    const ulonglong2* h = reinterpret_cast<const ulonglong2*>(a->hands + L.deal * 4);
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
    L.mode = a->mode;
    c->start_nodes = c->s.nodes;
    return true;
  }
  __device__ __forceinline__ int seed(const Lane& L) {
    return a->mode == MODE_STEP ? (int)a->seeds[L.deal * 20 + L.strain * 4 + L.decl] : 7;
  }
  __device__ __forceinline__ void answer(const Lane& L, int ns) {
    a->out20[L.deal * 20 + L.strain * 4 + L.decl] = (uint8_t)((L.decl & 1) == 0 ? ns : 13 - ns);
  }
  __device__ __forceinline__ void job_done(const Lane& L) {
    if (a->job_nodes) a->job_nodes[L.job] = c->s.nodes - c->start_nodes;
    if (a->job_end_ns) a->job_end_ns[L.job] = global_ns();
    c->jobs_done++;
  }
};

// Stage picked for the warp from the stages present: RET > NEXT > ROOT > TAKE > ENTER.
__device__ __forceinline__ int pick_stage(unsigned present) {
  if (present & (1u << ST_RET)) return ST_RET;
  if (present & (1u << ST_NEXT)) return ST_NEXT;
  if (present & (1u << ST_ROOT)) return ST_ROOT;
  if (present & (1u << ST_TAKE)) return ST_TAKE;
  return ST_ENTER;
}

// BLOCK threads per block; MINB resident blocks per SM asked of the register allocator.
// The lane's whole search state (position, top frame, search control) is in shared
// memory, so registers hold only the temporaries of the stage being run.
template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) batch_kernel(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BlockShared<BLOCK>& sh = *reinterpret_cast<BlockShared<BLOCK>*>(smem_raw);
  Lane* s_state = sh.lane;
  LaneCounters* s_lane = sh.cnt;
  auto& s_stage = sh.stage;
  const int tid = threadIdx.x, wid = tid >> 5, ln = tid & 31;
  const long long lane = (long long)blockIdx.x * BLOCK + tid;
  {
    memset(&s_lane[tid], 0, sizeof(LaneCounters));
    if (ln < 12) s_stage[wid][ln] = 0;
  }
  DevEnv env;
  env.a = &a;
  env.tt = a.tt + (lane << a.tt_log2);
  env.mask = (1u << a.tt_log2) - 1;
  env.stack = a.stacks + lane * STACK_DEPTH;
  env.c = &s_lane[tid];
  __syncwarp();

  Lane& L = s_state[tid];
  L.stage = ST_TAKE;
  L.sp = 0;
  L.gen = a.lane_gen[lane];
  L.v = 0;
  L.r = 0;
  L.p.trick = 0;
  unsigned iter = 0;
  for (;;) {
    const unsigned present = __reduce_or_sync(0xFFFFFFFFu, 1u << L.stage);
    if ((present & ~(1u << ST_IDLE)) == 0) break;
    if ((++iter & 4095u) == 0 && a.stop) {
      int stop = __shfl_sync(0xFFFFFFFFu, ln == 0 ? *a.stop : 0, 0);
      if (stop) {
        L.stage = ST_IDLE;  // unfinished results stay 255
        continue;
      }
    }
    const int pick = pick_stage(present);
    const bool run = L.stage == pick;
    const unsigned who = __ballot_sync(0xFFFFFFFFu, run);
    if (ln == 0) {
      s_stage[wid][pick]++;
      s_stage[wid][6 + pick] += __popc(who);
    }
    if (run) lane_step(L, env);
  }
  a.lane_gen[lane] = L.gen;
  __syncthreads();
  // Block sums of the counters, one atomic per word per block.
  if (tid < CNT_WORDS) {
    unsigned long long sum = 0;
    for (int t = 0; t < BLOCK; t++) {
      const LaneCounters& c = s_lane[t];
      switch (tid) {
        case CNT_NODES: sum += c.s.nodes; break;
        case CNT_PROBES: sum += c.s.tt.probes; break;
        case CNT_HITS: sum += c.s.tt.hits; break;
        case CNT_STORES: sum += c.s.tt.stores; break;
        case CNT_TT_BYTES: sum += c.s.tt.bytes; break;
        case CNT_JOBS_DONE: sum += c.jobs_done; break;
        default:
          if (tid >= CNT_EXIT && tid < CNT_EXIT + 7) sum += c.s.enter_exit[tid - CNT_EXIT];
      }
    }
    if (tid >= CNT_STAGE_ITERS && tid < CNT_STAGE_ITERS + 6)
      for (int w = 0; w < BLOCK / 32; w++) sum += s_stage[w][tid - CNT_STAGE_ITERS];
    if (tid >= CNT_STAGE_LANES && tid < CNT_STAGE_LANES + 6)
      for (int w = 0; w < BLOCK / 32; w++) sum += s_stage[w][6 + tid - CNT_STAGE_LANES];
    if (tid != CNT_NEXT_JOB && sum) atomicAdd(a.counters + tid, sum);
  }
}

}  // namespace ddg
