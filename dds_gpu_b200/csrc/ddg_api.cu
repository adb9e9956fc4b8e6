// C ABI of the solver (include/ddg.h): the device pool, the batch calls and the deal
// generator. Built with nvcc for sm_100a into libddg.so; there is no CPU path: without a
// CUDA device every solve call fails with DDG_E_CUDA.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <chrono>
#include <thread>
#include <vector>

#include "ddg.h"
#include "ddg_kernel.cuh"

using namespace ddg;

namespace {

thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

#define CUDA_TRY(x)                                                                          \
  do {                                                                                       \
    cudaError_t e_ = (x);                                                                    \
    if (e_ != cudaSuccess) return fail(DDG_E_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
  } while (0)

}  // namespace

struct KVariant;

struct ddg_solver {
  ddg_config cfg;
  int device = 0, lanes = 0, block = 128, sms = 0;
  const KVariant* variant = nullptr;
  TTBucket* tt = nullptr;
  Frame* stacks = nullptr;
  u32* lane_gen = nullptr;
  unsigned long long* counters = nullptr;
  int* h_stop = nullptr;
  int* d_stop = nullptr;
  size_t bytes = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // Staging buffers of the host-memory calls.
  uint64_t* d_hands = nullptr;
  uint8_t* d_out = nullptr;
  int8_t* d_seeds = nullptr;
  int64_t cap = 0;
  uint64_t total_nodes = 0;  // search nodes over all calls
  uint64_t* d_job_end_ns = nullptr;  // caller's buffer for job completion times, or null
  uint64_t start_ns = 0;             // device global timer at the last solve's launch
  TaskPool* tasks = nullptr;         // helping's task pool (cfg.help), cleared per solve
};

extern "C" {

const char* ddg_version(void) { return "ddg 0.1 (sm_100a)"; }
const char* ddg_last_error(void) { return g_err; }

void ddg_config_default(ddg_config* c) {
  memset(c, 0, sizeof(*c));
  c->tt_log2 = 10;
  c->lanes = 0;
  c->block = 128;
  c->jobs_per_deal = 5;
  c->device = 0;
  c->schedule = 0;
  c->time_limit_s = 0;
  c->mem_fraction = 0.85;
  c->help = 0;
}

int ddg_check_deal(const uint64_t* h) {
  if (!h) return fail(DDG_E_ARG, "null deal");
  const uint64_t valid = 0x1FFF1FFF1FFF1FFFull;
  uint64_t seen = 0;
  int n0 = __builtin_popcountll(h[0]);
  for (int i = 0; i < 4; i++) {
    if (h[i] & ~valid) return fail(DDG_E_ARG, "hand %d has bits outside the 52 cards", i);
    if (h[i] & seen) return fail(DDG_E_ARG, "hands overlap (hand %d)", i);
    if (__builtin_popcountll(h[i]) != n0) return fail(DDG_E_ARG, "hands differ in size");
    seen |= h[i];
  }
  if (n0 < 1 || n0 > 13) return fail(DDG_E_ARG, "hand size %d is not 1..13", n0);
  return DDG_OK;
}

// Compiled launch shapes: threads per block and the resident blocks per SM the register
// allocator is held to (1 = no limit beyond the block size).
typedef void (*BatchFn)(BatchArgs);
struct KVariant {
  int block, minb, schedule;
  BatchFn fn;
  size_t smem;  // dynamic shared memory per block
};
// schedule 0: block-phase kernel (all warps run each phase in turn); schedule 1: queue
// kernel (warps take lanes from per-phase queues, no block barriers).
#define DDG_VARIANT(B, M)                                     \
  {B, M, 0, batch_kernel<B, M>, sizeof(BlockShared<B>)}, { \
    B, M, 1, queue_kernel<B, M>, sizeof(BlockShared<B>)    \
  }
static const KVariant kVariants[] = {
    DDG_VARIANT(64, 1),  DDG_VARIANT(128, 1), DDG_VARIANT(128, 4), DDG_VARIANT(128, 6),
    DDG_VARIANT(256, 1), DDG_VARIANT(256, 2), DDG_VARIANT(256, 3),
};
#undef DDG_VARIANT

static const KVariant* find_variant(int block, int minb, int schedule) {
  if (minb <= 0) minb = 1;
  for (const KVariant& v : kVariants)
    if (v.block == block && v.minb == minb && v.schedule == schedule) return &v;
  return nullptr;
}

static int occupancy_blocks(const KVariant* v) {
  int nb = 0;
  cudaError_t e = cudaFuncSetAttribute((const void*)v->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v->smem);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, v->fn, v->block, v->smem);
  return e == cudaSuccess ? nb : 0;
}

void ddg_solver_destroy(ddg_solver* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  cudaFree(s->tt);
  cudaFree(s->stacks);
  cudaFree(s->lane_gen);
  cudaFree(s->counters);
  cudaFree(s->tasks);
  cudaFree(s->d_hands);
  cudaFree(s->d_out);
  cudaFree(s->d_seeds);
  if (s->h_stop) cudaFreeHost(s->h_stop);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  delete s;
}

int ddg_solver_create(const ddg_config* cfg_in, ddg_solver** out) {
  if (!out) return fail(DDG_E_ARG, "null output");
  *out = nullptr;
  ddg_config cfg;
  ddg_config_default(&cfg);
  if (cfg_in) {
    cfg = *cfg_in;
    if (!cfg.tt_log2) cfg.tt_log2 = 10;
    if (!cfg.block) cfg.block = 128;
    if (!cfg.jobs_per_deal) cfg.jobs_per_deal = 5;
    if (cfg.mem_fraction <= 0) cfg.mem_fraction = 0.85;
  }
  if (cfg.tt_log2 < TT_MIN_LOG2 || cfg.tt_log2 > 20)
    return fail(DDG_E_ARG, "tt_log2 %d is not in 9..20", cfg.tt_log2);
  if (cfg.schedule != 0 && cfg.schedule != 1) return fail(DDG_E_ARG, "schedule %d is not 0 or 1", cfg.schedule);
  const KVariant* variant = find_variant(cfg.block, cfg.min_blocks, cfg.schedule);
  if (!variant)
    return fail(DDG_E_ARG, "no kernel for block %d / min_blocks %d (64/1, 128/1,4,6, 256/1..3)", cfg.block,
                cfg.min_blocks);
  if (cfg.jobs_per_deal != 5 && cfg.jobs_per_deal != 20)
    return fail(DDG_E_ARG, "jobs_per_deal %d is not 5 or 20", cfg.jobs_per_deal);
  if (cfg.lanes < 0) return fail(DDG_E_ARG, "lanes %d < 0", cfg.lanes);
  int ndev = 0;
  CUDA_TRY(cudaGetDeviceCount(&ndev));
  if (cfg.device < 0 || cfg.device >= ndev) return fail(DDG_E_ARG, "device %d of %d", cfg.device, ndev);
  CUDA_TRY(cudaSetDevice(cfg.device));
  ddg_solver* s = new ddg_solver();
  s->cfg = cfg;
  s->device = cfg.device;
  s->block = cfg.block;
  s->variant = variant;
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, cfg.device);
  if (e != cudaSuccess) {
    delete s;
    return fail(DDG_E_CUDA, "cudaGetDeviceProperties: %s", cudaGetErrorString(e));
  }
  s->sms = prop.multiProcessorCount;
  const size_t per_lane = ((size_t)sizeof(TTBucket) << cfg.tt_log2) + sizeof(Frame) * STACK_DEPTH + 4;
  long long lanes = cfg.lanes;
  int nb = occupancy_blocks(variant);  // also sets the kernel's dynamic shared memory limit
  if (nb <= 0) {
    delete s;
    return fail(DDG_E_CUDA, "kernel variant %d/%d does not fit on an SM", cfg.block, cfg.min_blocks);
  }
  const long long resident = (long long)s->sms * nb * cfg.block;
  if (lanes == 0) lanes = resident;
  if (cfg.help && lanes > resident) {
    delete s;
    return fail(DDG_E_ARG, "helping needs every block resident: at most %lld lanes", resident);
  }
  size_t free_b = 0, total_b = 0;
  e = cudaMemGetInfo(&free_b, &total_b);
  if (e != cudaSuccess) {
    delete s;
    return fail(DDG_E_CUDA, "cudaMemGetInfo: %s", cudaGetErrorString(e));
  }
  const size_t budget = (size_t)((double)free_b * cfg.mem_fraction);
  if ((size_t)lanes * per_lane > budget) {
    if (cfg.lanes) {
      delete s;
      return fail(DDG_E_MEMORY, "%lld lanes need %.2f GB, %.2f GB free", lanes,
                  lanes * (double)per_lane / 1e9, free_b / 1e9);
    }
    lanes = (long long)(budget / per_lane);
  }
  lanes = lanes / cfg.block * cfg.block;
  if (lanes <= 0) {
    delete s;
    return fail(DDG_E_MEMORY, "no room for one block of lanes");
  }
  s->lanes = (int)lanes;
  size_t tt_bytes = (size_t)lanes * ((size_t)sizeof(TTBucket) << cfg.tt_log2);
  size_t st_bytes = (size_t)lanes * sizeof(Frame) * STACK_DEPTH;
  e = cudaMalloc(&s->tt, tt_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&s->stacks, st_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&s->lane_gen, (size_t)lanes * 4);
  if (e == cudaSuccess) e = cudaMalloc(&s->counters, CNT_WORDS * 8);
  if (e == cudaSuccess && cfg.help) e = cudaMalloc(&s->tasks, sizeof(TaskPool));
  if (e == cudaSuccess) e = cudaMemset(s->tt, 0, tt_bytes);
  if (e == cudaSuccess) e = cudaMemset(s->lane_gen, 0, (size_t)lanes * 4);
  if (e == cudaSuccess) e = cudaHostAlloc(&s->h_stop, sizeof(int), cudaHostAllocMapped);
  if (e == cudaSuccess) e = cudaHostGetDevicePointer((void**)&s->d_stop, s->h_stop, 0);
  if (e == cudaSuccess) e = cudaEventCreate(&s->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&s->ev1);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    ddg_solver_destroy(s);
    return fail(e == cudaErrorMemoryAllocation ? DDG_E_MEMORY : DDG_E_CUDA, "solver pool: %s",
                cudaGetErrorString(e));
  }
  *s->h_stop = 0;
  s->bytes = tt_bytes + st_bytes + (size_t)lanes * 4;
  *out = s;
  return DDG_OK;
}

int ddg_solver_lanes(const ddg_solver* s) { return s ? s->lanes : 0; }

int ddg_solver_set_job_times(ddg_solver* s, uint64_t* d_job_end_ns) {
  if (!s) return fail(DDG_E_ARG, "null solver");
  s->d_job_end_ns = d_job_end_ns;
  return DDG_OK;
}
uint64_t ddg_solver_nodes(const ddg_solver* s) { return s ? s->total_nodes : 0; }
int64_t ddg_solver_bytes(const ddg_solver* s) { return s ? (int64_t)s->bytes : 0; }

static int launch_batch(ddg_solver* s, const BatchArgs& a, long long n_jobs, cudaStream_t stream,
                        int* grid_out) {
  // With helping every resident lane is launched: lanes without a job help the others.
  long long want = (a.tasks || n_jobs > s->lanes) ? s->lanes : n_jobs;
  int grid = (int)((want + s->block - 1) / s->block);
  if (grid < 1) grid = 1;
  *grid_out = grid;
  BatchArgs args = a;
  void* params[] = {&args};
  CUDA_TRY(cudaLaunchKernel((const void*)s->variant->fn, dim3(grid), dim3(s->block), params, s->variant->smem,
                            stream));
  return DDG_OK;
}

int ddg_solve_device(ddg_solver* s, const uint64_t* d_hands, int64_t n, const int8_t* d_seed20,
                     uint8_t* d_out20, uint64_t* d_job_nodes, void* stream_v, ddg_stats* st) {
  if (!s) return fail(DDG_E_ARG, "null solver");
  if (n < 0 || (n > 0 && (!d_hands || !d_out20))) return fail(DDG_E_ARG, "bad batch arguments");
  if (st) memset(st, 0, sizeof(*st));
  if (n == 0) return DDG_OK;
  if ((reinterpret_cast<uintptr_t>(d_hands) & 15) != 0) return fail(DDG_E_ARG, "hands not 16-byte aligned");
  CUDA_TRY(cudaSetDevice(s->device));
  cudaStream_t stream = (cudaStream_t)stream_v;
  const int jpd = s->cfg.jobs_per_deal;
  const long long n_jobs = (long long)n * jpd;
  CUDA_TRY(cudaMemsetAsync(s->counters, 0, CNT_WORDS * 8, stream));
  CUDA_TRY(cudaMemsetAsync(d_out20, 0xFF, (size_t)n * 20, stream));
  *(volatile int*)s->h_stop = 0;
  BatchArgs a;
  a.hands = d_hands;
  a.n_jobs = n_jobs;
  a.jpd = jpd;
  a.mode = d_seed20 ? MODE_STEP : MODE_BISECT;
  a.seeds = d_seed20;
  a.out20 = d_out20;
  a.job_nodes = d_job_nodes;
  a.counters = s->counters;
  a.tt = s->tt;
  a.stacks = s->stacks;
  a.lane_gen = s->lane_gen;
  a.tt_log2 = s->cfg.tt_log2;
  a.schedule = s->cfg.schedule;
  a.stop = s->d_stop;
  a.job_end_ns = s->d_job_end_ns;
  a.tasks = s->tasks;
  a.free_below = s->cfg.free_below == 0 ? 64 : s->cfg.free_below < 0 ? 0 : s->cfg.free_below;
  a.free_steps = s->cfg.free_steps > 0 ? s->cfg.free_steps : 256;
  if (s->tasks) CUDA_TRY(cudaMemsetAsync(s->tasks, 0, sizeof(TaskPool), stream));
  if (s->d_job_end_ns) CUDA_TRY(cudaMemsetAsync(s->d_job_end_ns, 0, (size_t)n_jobs * 8, stream));
  CUDA_TRY(cudaEventRecord(s->ev0, stream));
  int grid = 0;
  int rc = launch_batch(s, a, n_jobs, stream, &grid);
  if (rc) return rc;
  CUDA_TRY(cudaEventRecord(s->ev1, stream));
  if (s->cfg.time_limit_s > 0) {
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
      cudaError_t q = cudaEventQuery(s->ev1);
      if (q == cudaSuccess) break;
      if (q != cudaErrorNotReady) return fail(DDG_E_CUDA, "solve kernel: %s", cudaGetErrorString(q));
      double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (el > s->cfg.time_limit_s) *(volatile int*)s->h_stop = 1;
      std::this_thread::sleep_for(std::chrono::milliseconds(2));
    }
  }
  CUDA_TRY(cudaEventSynchronize(s->ev1));
  CUDA_TRY(cudaGetLastError());
  unsigned long long c[CNT_WORDS];
  CUDA_TRY(cudaMemcpy(c, s->counters, sizeof(c), cudaMemcpyDeviceToHost));
  s->total_nodes += c[CNT_NODES];
  if (c[CNT_FAULTS])
    return fail(DDG_E_TIMEOUT, "%llu blocks gave up a bounded queue wait; results incomplete", c[CNT_FAULTS]);
  if (st) {
    st->nodes = c[CNT_NODES];
    st->tt_probes = c[CNT_PROBES];
    st->tt_hits = c[CNT_HITS];
    st->tt_stores = c[CNT_STORES];
    st->tt_bytes = c[CNT_TT_BYTES];
    for (int k = 0; k < 7; k++) st->enter_exit[k] = c[CNT_EXIT + k];
    for (int k = 0; k < PH_COUNT; k++) {
      st->phase_warps[k] = c[CNT_PHASE_WARPS + k];
      st->phase_items[k] = c[CNT_PHASE_ITEMS + k];
      st->phase_cycles[k] = c[CNT_PHASE_CYCLES + k];
    }
    st->free_rounds = c[CNT_PHASE_ITEMS + PH_COUNT];
    st->free_cycles = c[CNT_PHASE_CYCLES + PH_COUNT];
    st->iterations = c[CNT_ITERS];
    st->tasks = 0;
    if (s->tasks) {
      int posted = 0;
      CUDA_TRY(cudaMemcpy(&posted, &s->tasks->posted, sizeof(int), cudaMemcpyDeviceToHost));
      st->tasks = (uint64_t)posted;
    }
    st->jobs_done = (int64_t)c[CNT_JOBS_DONE];
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    st->kernel_ms = ms;
    st->grid = grid;
    st->block = s->block;
    st->lanes = grid * s->block;
  }
  return DDG_OK;
}

static int ensure_staging(ddg_solver* s, int64_t n) {
  if (n <= s->cap) return DDG_OK;
  cudaFree(s->d_hands);
  cudaFree(s->d_out);
  cudaFree(s->d_seeds);
  s->d_hands = nullptr;
  s->d_out = nullptr;
  s->d_seeds = nullptr;
  s->cap = 0;
  CUDA_TRY(cudaMalloc(&s->d_hands, (size_t)n * 32));
  CUDA_TRY(cudaMalloc(&s->d_out, (size_t)n * 20));
  CUDA_TRY(cudaMalloc(&s->d_seeds, (size_t)n * 20));
  s->cap = n;
  return DDG_OK;
}

static int solve_host(ddg_solver* s, const uint64_t* hands, int64_t n, const int8_t* seeds,
                      uint8_t* out20, ddg_stats* st) {
  if (!s) return fail(DDG_E_ARG, "null solver");
  if (n < 0 || (n > 0 && (!hands || !out20))) return fail(DDG_E_ARG, "bad batch arguments");
  if (st) memset(st, 0, sizeof(*st));
  if (n == 0) return DDG_OK;
  for (int64_t i = 0; i < n; i++) {
    int rc = ddg_check_deal(hands + i * 4);
    if (rc) return fail(rc, "deal %lld: %s", (long long)i, g_err);
  }
  CUDA_TRY(cudaSetDevice(s->device));
  int rc = ensure_staging(s, n);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpy(s->d_hands, hands, (size_t)n * 32, cudaMemcpyHostToDevice));
  if (seeds) CUDA_TRY(cudaMemcpy(s->d_seeds, seeds, (size_t)n * 20, cudaMemcpyHostToDevice));
  rc = ddg_solve_device(s, s->d_hands, n, seeds ? s->d_seeds : nullptr, s->d_out, nullptr, nullptr, st);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpy(out20, s->d_out, (size_t)n * 20, cudaMemcpyDeviceToHost));
  return DDG_OK;
}

int ddg_solve_batch(ddg_solver* s, const uint64_t* hands, int64_t n, uint8_t* out20, ddg_stats* st) {
  return solve_host(s, hands, n, nullptr, out20, st);
}

int ddg_solve_batch_seeded(ddg_solver* s, const uint64_t* hands, int64_t n, const int8_t* ns_seed20,
                           uint8_t* out20, ddg_stats* st) {
  if (!ns_seed20) return fail(DDG_E_ARG, "null seeds");
  return solve_host(s, hands, n, ns_seed20, out20, st);
}

int ddg_solve_strain(ddg_solver* s, const uint64_t* hands4, int strain, const int* ns4, int* out4) {
  if (strain < 0 || strain > 4) return fail(DDG_E_ARG, "strain %d is not 0..4", strain);
  if (!out4) return fail(DDG_E_ARG, "null output");
  int8_t seeds[20];
  for (int i = 0; i < 20; i++) seeds[i] = 7;
  if (ns4)
    for (int d = 0; d < 4; d++) seeds[strain * 4 + d] = (int8_t)ns4[d];
  uint8_t out[20];
  // One deal: all five strains are solved; the batch form amortises this.
  int rc = solve_host(s, hands4, 1, ns4 ? seeds : nullptr, out, nullptr);
  if (rc) return rc;
  for (int d = 0; d < 4; d++) out4[d] = out[strain * 4 + d];
  return DDG_OK;
}

static inline uint64_t splitmix_next(uint64_t& x) {
  x += 0x9E3779B97F4A7C15ull;
  uint64_t z = x;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

void ddg_make_deals(uint64_t seed, int64_t first, int64_t n, int k, uint64_t* hands) {
  if (k < 1) k = 1;
  if (k > 13) k = 13;
  for (int64_t d = 0; d < n; d++) {
    uint64_t x = seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(first + d + 1));
    int cards[52];
    for (int i = 0; i < 52; i++) cards[i] = (i / 13) * 16 + i % 13;
    for (int i = 51; i > 0; i--) {
      int j = (int)(splitmix_next(x) % (uint64_t)(i + 1));
      int t = cards[i];
      cards[i] = cards[j];
      cards[j] = t;
    }
    uint64_t* h = hands + d * 4;
    h[0] = h[1] = h[2] = h[3] = 0;
    for (int i = 0; i < 4 * k; i++) h[i % 4] |= 1ull << cards[i];
  }
}

}  // extern "C"
