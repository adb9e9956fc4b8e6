// C ABI of the solver (include/ddg.h): the device pool, the batch calls and the deal
// generator. Built with nvcc for sm_100a into libddg.so; there is no CPU path: without a
// CUDA device every solve call fails with DDG_E_CUDA.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <mutex>
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
  uint64_t* d_job_start_ns = nullptr;  // caller's buffer for the times jobs were taken, or null
  uint64_t start_ns = 0;             // device global timer at the last solve's launch
  TaskPool* tasks = nullptr;         // helping's task pool (cfg.help), cleared per solve
  size_t tasks_bytes = 0;            // the pool and, after it, one TT-user count per lane
  // Resumable (time-sliced) solve.
  LaneSave* save = nullptr;  // lanes x LaneSave, allocated by the first ddg_solve_begin
  BatchArgs slice_args;
  int64_t slice_n = 0;
  bool sliced = false, slice_done = false;
  bool streaming = false;  // a ddg_stream owns the lanes until it is closed
  // CUDA graph of one batch solve (ddg_solve_graph): rebuilt when its arguments change.
  cudaGraphExec_t graph = nullptr;
  const void* graph_key[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  int64_t graph_n = -1;
  int graph_grid = 0;
};

extern "C" {

#if defined(DDG_BOUNDS_CHECK)
const char* ddg_version(void) { return "ddg 0.2 (sm_100a, bounds-checked)"; }
#elif defined(DDG_TT_SIG)
const char* ddg_version(void) { return "ddg 0.2 (sm_100a, 12-byte signature TT entries, not strictly exact)"; }
#else
const char* ddg_version(void) { return "ddg 0.2 (sm_100a)"; }
#endif
const char* ddg_last_error(void) { return g_err; }

void ddg_config_default(ddg_config* c) {
  memset(c, 0, sizeof(*c));
  c->tt_log2 = 10;
  c->lanes = 0;
  c->block = 512;
  c->min_blocks = 1;
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
    DDG_VARIANT(256, 1), DDG_VARIANT(256, 2), DDG_VARIANT(256, 3), DDG_VARIANT(512, 1),
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
  cudaFree(s->save);
  if (s->graph) cudaGraphExecDestroy(s->graph);
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
    if (!cfg.block) cfg.block = 512;
    if (!cfg.min_blocks) cfg.min_blocks = cfg.block == 256 ? 2 : 1;  // the measured best shape
    if (!cfg.jobs_per_deal) cfg.jobs_per_deal = 5;
    if (cfg.mem_fraction <= 0) cfg.mem_fraction = 0.85;
  }
  if (cfg.tt_log2 < TT_MIN_LOG2 || cfg.tt_log2 > 20)
    return fail(DDG_E_ARG, "tt_log2 %d is not in 9..20", cfg.tt_log2);
  if (cfg.schedule < 0 || cfg.schedule > 2) return fail(DDG_E_ARG, "schedule %d is not 0, 1 or 2", cfg.schedule);
  const KVariant* variant = find_variant(cfg.block, cfg.min_blocks, cfg.schedule == 1 ? 1 : 0);
  if (!variant)
    return fail(DDG_E_ARG, "no kernel for block %d / min_blocks %d (64/1, 128/1,4,6, 256/1..3, 512/1)", cfg.block,
                cfg.min_blocks);
  if (cfg.jobs_per_deal != 5 && cfg.jobs_per_deal != 20)
    return fail(DDG_E_ARG, "jobs_per_deal %d is not 5 or 20", cfg.jobs_per_deal);
  if (cfg.lanes < 0) return fail(DDG_E_ARG, "lanes %d < 0", cfg.lanes);
  if (cfg.free_pack < 0 || cfg.free_pack > 32) return fail(DDG_E_ARG, "free_pack %d is not 0..32", cfg.free_pack);
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
  s->tasks_bytes = (sizeof(TaskPool) + 255) / 256 * 256 + (size_t)lanes * sizeof(int);
  if (e == cudaSuccess && cfg.help) e = cudaMalloc(&s->tasks, s->tasks_bytes);
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

int ddg_solver_set_job_starts(ddg_solver* s, uint64_t* d_job_start_ns) {
  if (!s) return fail(DDG_E_ARG, "null solver");
  s->d_job_start_ns = d_job_start_ns;
  return DDG_OK;
}
uint64_t ddg_solver_nodes(const ddg_solver* s) { return s ? s->total_nodes : 0; }
int64_t ddg_solver_bytes(const ddg_solver* s) { return s ? (int64_t)s->bytes : 0; }

static int launch_batch(ddg_solver* s, const BatchArgs& a, long long n_jobs, cudaStream_t stream,
                        int* grid_out) {
  // Every lane is launched: the first jobs are dealt round-robin over the blocks, so a small
  // batch spreads over all SMs (lanes without a job end at once, or help with helping on).
  (void)n_jobs;
  int grid = (int)((s->lanes + s->block - 1) / s->block);
  if (grid < 1) grid = 1;
  *grid_out = grid;
  BatchArgs args = a;
  const long long lanes = (long long)grid * s->block;
  args.rr_jobs = a.ring ? 0 : (a.n_jobs < lanes ? a.n_jobs : lanes);
  void* params[] = {&args};
  CUDA_TRY(cudaLaunchKernel((const void*)s->variant->fn, dim3(grid), dim3(s->block), params, s->variant->smem,
                            stream));
  return DDG_OK;
}

static BatchArgs make_args(ddg_solver* s, const uint64_t* d_hands, int64_t n, const int8_t* d_seed20,
                           uint8_t* d_out20, uint64_t* d_job_nodes) {
  BatchArgs a;
  memset(&a, 0, sizeof(a));
  const int jpd = s->cfg.jobs_per_deal;
  a.hands = d_hands;
  a.n_jobs = (long long)n * jpd;
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
  a.job_start_ns = s->d_job_start_ns;
  a.tasks = s->tasks;
  a.share_tt = s->tasks && s->cfg.help_share_tt >= 0;  // 0 = the default: shared
  a.tt_users = s->tasks ? reinterpret_cast<int*>(reinterpret_cast<char*>(s->tasks) + (sizeof(TaskPool) + 255) / 256 * 256)
                        : nullptr;
  a.free_below = s->cfg.free_below == 0 ? 96 : s->cfg.free_below < 0 ? 0 : s->cfg.free_below;
  a.free_steps = s->cfg.free_steps > 0 ? s->cfg.free_steps : 256;
  a.next_job = s->counters + CNT_NEXT_JOB;
  a.spread = s->cfg.phase_spread;
  a.cheap_limit = s->cfg.cheap_limit == 0 ? 3 : s->cfg.cheap_limit < 0 ? 0 : s->cfg.cheap_limit;
  a.fuse_follow = s->cfg.schedule == 2;
  a.flat_moves = s->cfg.flat_moves >= 0;  // 0 = the default: flattened
  a.free_pack = s->cfg.free_pack;  // 0: by the block's busy lanes
  return a;
}

// Counters of the last launch into `st` (and the solver's node total). Returns the words.
static int read_stats(ddg_solver* s, int grid, ddg_stats* st, unsigned long long* c) {
  CUDA_TRY(cudaMemcpy(c, s->counters, CNT_WORDS * 8, cudaMemcpyDeviceToHost));
  s->total_nodes += c[CNT_NODES];
  if (c[CNT_FAULTS])
    return fail(DDG_E_TIMEOUT, "%llu blocks gave up a bounded queue wait; results incomplete", c[CNT_FAULTS]);
  if (c[CNT_BOUNDS])
    return fail(DDG_E_STATE, "bounds check: %llu out-of-range accesses were skipped; results incomplete",
                c[CNT_BOUNDS]);
  if (!st) return DDG_OK;
  st->nodes = c[CNT_NODES];
  st->tt_probes = c[CNT_PROBES];
  st->tt_hits = c[CNT_HITS];
  st->tt_stores = c[CNT_STORES];
  st->tt_bytes = c[CNT_TT_BYTES];
  st->tt_entry_reads = c[CNT_ENTRY_READS];
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
  return DDG_OK;
}

// Waits for the launch between ev0 and ev1; the host time limit raises the stop flag.
static int wait_launch(ddg_solver* s) {
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
  return DDG_OK;
}

int ddg_solve_device(ddg_solver* s, const uint64_t* d_hands, int64_t n, const int8_t* d_seed20,
                     uint8_t* d_out20, uint64_t* d_job_nodes, void* stream_v, ddg_stats* st) {
  return ddg_solve_device_ex(s, d_hands, n, d_seed20, nullptr, d_out20, nullptr, d_job_nodes, stream_v, st);
}

int ddg_solve_device_ex(ddg_solver* s, const uint64_t* d_hands, int64_t n, const int8_t* d_seed20,
                        const int8_t* d_hint20, uint8_t* d_out20, int8_t* d_best20, uint64_t* d_job_nodes,
                        void* stream_v, ddg_stats* st) {
  if (!s) return fail(DDG_E_ARG, "null solver");
  if (n < 0 || (n > 0 && (!d_hands || !d_out20))) return fail(DDG_E_ARG, "bad batch arguments");
  if (st) memset(st, 0, sizeof(*st));
  if (n == 0) return DDG_OK;
  if ((reinterpret_cast<uintptr_t>(d_hands) & 15) != 0) return fail(DDG_E_ARG, "hands not 16-byte aligned");
  if (s->streaming) return fail(DDG_E_STATE, "a stream is open on this solver");
  CUDA_TRY(cudaSetDevice(s->device));
  s->sliced = false;  // a plain solve ends any resumable one
  cudaStream_t stream = (cudaStream_t)stream_v;
  BatchArgs a = make_args(s, d_hands, n, d_seed20, d_out20, d_job_nodes);
  a.hint20 = d_hint20;
  a.best20 = d_best20;
  CUDA_TRY(cudaMemsetAsync(s->counters, 0, CNT_WORDS * 8, stream));
  CUDA_TRY(cudaMemsetAsync(d_out20, 0xFF, (size_t)n * 20, stream));
  if (d_best20) CUDA_TRY(cudaMemsetAsync(d_best20, 0xFF, (size_t)n * 20, stream));
  *(volatile int*)s->h_stop = 0;
  if (s->tasks) CUDA_TRY(cudaMemsetAsync(s->tasks, 0, s->tasks_bytes, stream));
  if (s->d_job_end_ns) CUDA_TRY(cudaMemsetAsync(s->d_job_end_ns, 0, (size_t)a.n_jobs * 8, stream));
  if (s->d_job_start_ns) CUDA_TRY(cudaMemsetAsync(s->d_job_start_ns, 0, (size_t)a.n_jobs * 8, stream));
  CUDA_TRY(cudaEventRecord(s->ev0, stream));
  int grid = 0;
  int rc = launch_batch(s, a, a.n_jobs, stream, &grid);
  if (rc) return rc;
  CUDA_TRY(cudaEventRecord(s->ev1, stream));
  rc = wait_launch(s);
  if (rc) return rc;
  unsigned long long c[CNT_WORDS];
  return read_stats(s, grid, st, c);
}

int ddg_solve_graph(ddg_solver* s, const uint64_t* d_hands, int64_t n, const int8_t* d_seed20, uint8_t* d_out20,
                    void* stream_v, ddg_stats* st) {
  if (!s) return fail(DDG_E_ARG, "null solver");
  if (n <= 0 || !d_hands || !d_out20) return fail(DDG_E_ARG, "bad batch arguments");
  if ((reinterpret_cast<uintptr_t>(d_hands) & 15) != 0) return fail(DDG_E_ARG, "hands not 16-byte aligned");
  if (s->streaming) return fail(DDG_E_STATE, "a stream is open on this solver");
  if (st) memset(st, 0, sizeof(*st));
  CUDA_TRY(cudaSetDevice(s->device));
  s->sliced = false;
  cudaStream_t stream = (cudaStream_t)stream_v;
  const bool same = s->graph && s->graph_n == n && s->graph_key[0] == d_hands && s->graph_key[1] == d_seed20 &&
                    s->graph_key[2] == d_out20 && s->graph_key[3] == s->d_job_end_ns &&
                    s->graph_key[4] == s->d_job_start_ns;
  if (!same) {
    if (s->graph) cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
    // The solve as one graph: clear the counters, the tables, the task pool, launch.
    cudaStream_t cap = nullptr;
    CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    BatchArgs a = make_args(s, d_hands, n, d_seed20, d_out20, nullptr);
    a.job_end_ns = s->d_job_end_ns;
    a.job_start_ns = s->d_job_start_ns;
    cudaGraph_t g = nullptr;
    int grid = 0, rc = DDG_OK;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->counters, 0, CNT_WORDS * 8, cap);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_out20, 0xFF, (size_t)n * 20, cap);
    if (e == cudaSuccess && s->tasks) e = cudaMemsetAsync(s->tasks, 0, s->tasks_bytes, cap);
    if (e == cudaSuccess && s->d_job_end_ns) e = cudaMemsetAsync(s->d_job_end_ns, 0, (size_t)a.n_jobs * 8, cap);
    if (e == cudaSuccess && s->d_job_start_ns)
      e = cudaMemsetAsync(s->d_job_start_ns, 0, (size_t)a.n_jobs * 8, cap);
    if (e == cudaSuccess) rc = launch_batch(s, a, a.n_jobs, cap, &grid);
    cudaError_t e2 = cudaStreamEndCapture(cap, &g);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess && rc == DDG_OK) e = cudaGraphInstantiate(&s->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cap);
    if (rc) return rc;
    if (e != cudaSuccess) {
      s->graph = nullptr;
      return fail(DDG_E_CUDA, "solve graph: %s", cudaGetErrorString(e));
    }
    s->graph_n = n;
    s->graph_key[0] = d_hands;
    s->graph_key[1] = d_seed20;
    s->graph_key[2] = d_out20;
    s->graph_key[3] = s->d_job_end_ns;
    s->graph_key[4] = s->d_job_start_ns;
    s->graph_grid = grid;
  }
  *(volatile int*)s->h_stop = 0;
  CUDA_TRY(cudaEventRecord(s->ev0, stream));
  CUDA_TRY(cudaGraphLaunch(s->graph, stream));
  CUDA_TRY(cudaEventRecord(s->ev1, stream));
  int rc = wait_launch(s);
  if (rc) return rc;
  unsigned long long c[CNT_WORDS];
  return read_stats(s, s->graph_grid, st, c);
}

int ddg_solve_begin(ddg_solver* s, const uint64_t* d_hands, int64_t n, const int8_t* d_seed20, uint8_t* d_out20,
                    void* stream_v) {
  return ddg_solve_begin_ex(s, d_hands, n, d_seed20, nullptr, d_out20, stream_v);
}

int ddg_solve_begin_ex(ddg_solver* s, const uint64_t* d_hands, int64_t n, const int8_t* d_seed20,
                       const int8_t* d_hint20, uint8_t* d_out20, void* stream_v) {
  if (!s) return fail(DDG_E_ARG, "null solver");
  if (n <= 0 || !d_hands || !d_out20) return fail(DDG_E_ARG, "bad batch arguments");
  if ((reinterpret_cast<uintptr_t>(d_hands) & 15) != 0) return fail(DDG_E_ARG, "hands not 16-byte aligned");
  if (s->streaming) return fail(DDG_E_STATE, "a stream is open on this solver");
  CUDA_TRY(cudaSetDevice(s->device));
  if (!s->save) {
    cudaError_t e = cudaMalloc(&s->save, (size_t)s->lanes * sizeof(LaneSave));
    if (e != cudaSuccess) {
      s->save = nullptr;
      return fail(e == cudaErrorMemoryAllocation ? DDG_E_MEMORY : DDG_E_CUDA, "lane save area: %s",
                  cudaGetErrorString(e));
    }
    s->bytes += (size_t)s->lanes * sizeof(LaneSave);
  }
  cudaStream_t stream = (cudaStream_t)stream_v;
  s->slice_args = make_args(s, d_hands, n, d_seed20, d_out20, nullptr);
  s->slice_args.hint20 = d_hint20;
  s->slice_args.save = s->save;
  s->slice_args.resume = 0;
  s->slice_n = n;
  CUDA_TRY(cudaMemsetAsync(s->counters, 0, CNT_WORDS * 8, stream));
  CUDA_TRY(cudaMemsetAsync(d_out20, 0xFF, (size_t)n * 20, stream));
  if (s->tasks) CUDA_TRY(cudaMemsetAsync(s->tasks, 0, s->tasks_bytes, stream));
  if (s->d_job_end_ns) CUDA_TRY(cudaMemsetAsync(s->d_job_end_ns, 0, (size_t)s->slice_args.n_jobs * 8, stream));
  if (s->d_job_start_ns)
    CUDA_TRY(cudaMemsetAsync(s->d_job_start_ns, 0, (size_t)s->slice_args.n_jobs * 8, stream));
  s->sliced = true;
  s->slice_done = false;
  return DDG_OK;
}

int ddg_solve_continue(ddg_solver* s, double seconds, const uint64_t* hands_host, uint8_t* out20_host,
                       void* stream_v, ddg_stats* st, int* finished) {
  if (!s) return fail(DDG_E_ARG, "null solver");
  if (st) memset(st, 0, sizeof(*st));
  if (finished) *finished = 0;
  if (!s->sliced) return fail(DDG_E_STATE, "no resumable solve: call ddg_solve_begin first");
  if (!(seconds > 0)) return fail(DDG_E_ARG, "slice of %g s", seconds);
  CUDA_TRY(cudaSetDevice(s->device));
  cudaStream_t stream = (cudaStream_t)stream_v;
  BatchArgs a = s->slice_args;
  CUDA_TRY(cudaEventRecord(s->ev0, stream));
  if (hands_host)  // the caller's deals again (pinned memory makes this an async copy)
    CUDA_TRY(cudaMemcpyAsync((void*)a.hands, hands_host, (size_t)s->slice_n * 32, cudaMemcpyHostToDevice, stream));
  int grid = 0;
  if (!s->slice_done) {
    // Every counter but the job queue's head starts again at zero.
    CUDA_TRY(cudaMemsetAsync(s->counters + 1, 0, (CNT_WORDS - 1) * 8, stream));
    *(volatile int*)s->h_stop = 0;
    a.slice_ns = (u64)(seconds * 1e9);
    int rc = launch_batch(s, a, a.n_jobs, stream, &grid);
    if (rc) return rc;
  }
  if (out20_host)
    CUDA_TRY(cudaMemcpyAsync(out20_host, a.out20, (size_t)s->slice_n * 20, cudaMemcpyDeviceToHost, stream));
  CUDA_TRY(cudaEventRecord(s->ev1, stream));
  int rc = wait_launch(s);
  if (rc) return rc;
  if (s->slice_done) {
    if (finished) *finished = 1;
    return DDG_OK;
  }
  s->slice_args.resume = 1;
  unsigned long long c[CNT_WORDS];
  rc = read_stats(s, grid, st, c);
  if (rc) return rc;
  if ((long long)c[CNT_BLOCKS_DONE] == grid) s->slice_done = true;
  if (finished) *finished = s->slice_done ? 1 : 0;
  return DDG_OK;
}


// ---- streams: a device ring of deals fed while the persistent kernel runs ---------------

// The guide's inference on `stream` (ddg_guide_api.cuh): seeds and root leads of n deals.
static int guide_predict_on(ddg_guide* g, const uint64_t* d_hands, int64_t n, int8_t* d_seed20, int8_t* d_hint20,
                            cudaStream_t stream);

struct ddg_stream {
  ddg_solver* s = nullptr;
  int slots = 0;
  long long admit = 0;  // most deals in flight (published, not yet polled)
  u64* d_ring = nullptr;
  uint8_t* d_out = nullptr;
  int* d_done = nullptr;
  unsigned long long* d_words = nullptr;  // [0] published, [1] next job, [2] completion tail, [3] closing
  CompRec* h_comp = nullptr;              // mapped host memory
  CompRec* d_comp = nullptr;
  u64* h_stage = nullptr;                 // pinned mirror of the ring
  unsigned long long* h_words = nullptr;  // pinned sources of the published / closing words
  std::vector<uint8_t> slot_busy;
  unsigned long long published = 0, consumed = 0;
  cudaStream_t kstream = nullptr, cstream = nullptr;
  cudaEvent_t kdone = nullptr;
  ddg_guide* guide = nullptr;             // guided stream: seeds and root leads per ring slot
  int8_t* d_seed = nullptr;
  int8_t* d_hint = nullptr;
  bool launched = false;
  double idle_timeout_s = 30;
  int launches = 0;
};

static void stream_free(ddg_stream* st) {
  if (!st) return;
  if (st->kstream) cudaStreamSynchronize(st->kstream);
  cudaFree(st->d_ring);
  cudaFree(st->d_out);
  cudaFree(st->d_done);
  cudaFree(st->d_seed);
  cudaFree(st->d_hint);
  cudaFree(st->d_words);
  if (st->h_comp) cudaFreeHost(st->h_comp);
  if (st->h_stage) cudaFreeHost(st->h_stage);
  if (st->h_words) cudaFreeHost(st->h_words);
  if (st->kstream) cudaStreamDestroy(st->kstream);
  if (st->cstream) cudaStreamDestroy(st->cstream);
  if (st->kdone) cudaEventDestroy(st->kdone);
  if (st->s) st->s->streaming = false;
  delete st;
}

// Launches the stream kernel unless it is running; it ends by itself once its lanes found
// no deal for idle_timeout_s, or once the stream is closing and every deal is done.
static int stream_kernel(ddg_stream* st) {
  if (st->launched) {
    cudaError_t q = cudaEventQuery(st->kdone);
    if (q == cudaErrorNotReady) return DDG_OK;
    if (q != cudaSuccess) return fail(DDG_E_CUDA, "stream kernel: %s", cudaGetErrorString(q));
    st->launched = false;
    unsigned long long faults = 0;
    CUDA_TRY(cudaMemcpy(&faults, st->s->counters + CNT_FAULTS, 8, cudaMemcpyDeviceToHost));
    if (faults) return fail(DDG_E_TIMEOUT, "stream kernel gave up a bounded wait");
  }
  ddg_solver* s = st->s;
  BatchArgs a = make_args(s, nullptr, 0, nullptr, st->d_out, nullptr);
  a.tasks = nullptr;  // lanes without a deal wait for the next one instead of helping
  a.job_end_ns = nullptr;
  a.job_start_ns = nullptr;
  a.ring = st->d_ring;
  a.published = st->d_words + 0;
  a.next_job = st->d_words + 1;
  a.comp_tail = st->d_words + 2;
  a.closing = reinterpret_cast<const int*>(st->d_words + 3);
  a.deal_done = st->d_done;
  a.comp = st->d_comp;
  a.ring_mask = st->slots - 1;
  a.idle_ns = (u64)(st->idle_timeout_s * 1e9);
  a.n_jobs = 0;
  if (st->guide) {  // each slot's NS seeds (stepping search) and root leads, written at submit
    a.mode = MODE_STEP;
    a.seeds = st->d_seed;
    a.hint20 = st->d_hint;
  }
  *(volatile int*)s->h_stop = 0;
  int grid = 0;
  int rc = launch_batch(s, a, (long long)s->lanes, st->kstream, &grid);
  if (rc) return rc;
  CUDA_TRY(cudaEventRecord(st->kdone, st->kstream));
  st->launched = true;
  st->launches++;
  return DDG_OK;
}

int ddg_stream_open(ddg_solver* s, int ring_slots, double idle_timeout_s, ddg_stream** out) {
  return ddg_stream_open_guided(s, ring_slots, idle_timeout_s, nullptr, out);
}

int ddg_stream_open_guided(ddg_solver* s, int ring_slots, double idle_timeout_s, ddg_guide* guide,
                           ddg_stream** out) {
  if (!out) return fail(DDG_E_ARG, "null output");
  *out = nullptr;
  if (!s) return fail(DDG_E_ARG, "null solver");
  if (guide && (s->lanes + s->block - 1) / s->block > s->sms - 2)
    return fail(DDG_E_STATE,
                "a guided stream needs SMs the solver leaves free for the guide's kernels: create the solver "
                "with lanes <= (SMs - 2) * block = %d",
                (s->sms - 2) * s->block);
  if (s->streaming) return fail(DDG_E_STATE, "a stream is already open on this solver");
  if (s->cfg.schedule == 1) return fail(DDG_E_ARG, "streams run on the block-phase kernel (schedule 0 or 2)");
  if (ring_slots <= 0) ring_slots = 65536;
  if (ring_slots < 64 || ring_slots > (1 << 22) || (ring_slots & (ring_slots - 1)))
    return fail(DDG_E_ARG, "ring_slots %d is not a power of two in 64..4M", ring_slots);
  CUDA_TRY(cudaSetDevice(s->device));
  ddg_stream* st = new ddg_stream();
  st->s = s;
  st->slots = ring_slots;
  st->idle_timeout_s = idle_timeout_s > 0 ? idle_timeout_s : 30;
  // Admission by TT memory: a deal's jobs each need a lane (and its TT); at most two jobs
  // per lane are admitted, one running and one waiting.
  st->admit = (long long)s->lanes * 2 / s->cfg.jobs_per_deal;
  if (st->admit > ring_slots) st->admit = ring_slots;
  if (st->admit < 1) st->admit = 1;
  st->slot_busy.assign(ring_slots, 0);
  s->streaming = true;
  cudaError_t e = cudaMalloc(&st->d_ring, (size_t)ring_slots * 32);
  if (e == cudaSuccess) e = cudaMalloc(&st->d_out, (size_t)ring_slots * 20);
  if (e == cudaSuccess) e = cudaMalloc(&st->d_done, (size_t)ring_slots * 4);
  if (e == cudaSuccess) e = cudaMalloc(&st->d_words, 4 * 8);
  if (e == cudaSuccess) e = cudaHostAlloc(&st->h_comp, (size_t)ring_slots * sizeof(CompRec), cudaHostAllocMapped);
  if (e == cudaSuccess) e = cudaHostGetDevicePointer((void**)&st->d_comp, st->h_comp, 0);
  if (e == cudaSuccess) e = cudaHostAlloc(&st->h_stage, (size_t)ring_slots * 32, cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaHostAlloc(&st->h_words, 4 * 8, cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st->kstream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st->cstream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st->kdone, cudaEventDisableTiming);
  if (e == cudaSuccess && guide) {
    st->guide = guide;
    e = cudaMalloc(&st->d_seed, (size_t)ring_slots * 20);
    if (e == cudaSuccess) e = cudaMalloc(&st->d_hint, (size_t)ring_slots * 20);
  }
  if (e == cudaSuccess) e = cudaMemset(st->d_done, 0, (size_t)ring_slots * 4);
  if (e == cudaSuccess) e = cudaMemset(st->d_words, 0, 4 * 8);
  if (e == cudaSuccess) e = cudaMemset(s->counters, 0, CNT_WORDS * 8);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    stream_free(st);
    return fail(e == cudaErrorMemoryAllocation ? DDG_E_MEMORY : DDG_E_CUDA, "stream buffers: %s",
                cudaGetErrorString(e));
  }
  memset(st->h_comp, 0, (size_t)ring_slots * sizeof(CompRec));
  int rc = stream_kernel(st);
  if (rc) {
    stream_free(st);
    return rc;
  }
  *out = st;
  return DDG_OK;
}

int64_t ddg_stream_capacity(const ddg_stream* st) { return st ? st->admit : 0; }
int64_t ddg_stream_in_flight(const ddg_stream* st) { return st ? (int64_t)(st->published - st->consumed) : 0; }

int ddg_stream_submit(ddg_stream* st, const uint64_t* hands, int64_t n, int64_t* accepted) {
  if (accepted) *accepted = 0;
  if (!st) return fail(DDG_E_ARG, "null stream");
  if (n < 0 || (n > 0 && !hands)) return fail(DDG_E_ARG, "bad submit arguments");
  for (int64_t i = 0; i < n; i++) {
    int rc = ddg_check_deal(hands + i * 4);
    if (rc) return fail(rc, "deal %lld: %s", (long long)i, g_err);
  }
  CUDA_TRY(cudaSetDevice(st->s->device));
  const unsigned long long mask = (unsigned long long)st->slots - 1;
  // Admission: ring slots and TT memory; a slot is reused only after its deal was polled.
  int64_t k = 0;
  while (k < n && (long long)(st->published + k - st->consumed) < st->admit &&
         !st->slot_busy[(st->published + k) & mask])
    k++;
  if (k > 0) {
    const unsigned long long first = st->published & mask;
    for (int64_t i = 0; i < k; i++) {
      const unsigned long long slot = (st->published + i) & mask;
      memcpy(st->h_stage + slot * 4, hands + i * 4, 32);
      st->slot_busy[slot] = 1;
    }
    const unsigned long long run1 = std::min<unsigned long long>((unsigned long long)k, st->slots - first);
    CUDA_TRY(cudaMemcpyAsync(st->d_ring + first * 4, st->h_stage + first * 4, run1 * 32, cudaMemcpyHostToDevice,
                             st->cstream));
    if ((unsigned long long)k > run1)
      CUDA_TRY(cudaMemcpyAsync(st->d_ring, st->h_stage, (k - run1) * 32, cudaMemcpyHostToDevice, st->cstream));
    if (st->guide) {  // the guide's seeds and leads for the new slots, before they are published
      int rc = guide_predict_on(st->guide, st->d_ring + first * 4, (int64_t)run1, st->d_seed + first * 20,
                                st->d_hint + first * 20, st->cstream);
      if (rc == DDG_OK && (unsigned long long)k > run1)
        rc = guide_predict_on(st->guide, st->d_ring, (int64_t)(k - run1), st->d_seed, st->d_hint, st->cstream);
      if (rc) {
        for (int64_t i = 0; i < k; i++) st->slot_busy[(st->published + i) & mask] = 0;
        return rc;
      }
    }
    st->h_words[0] = st->published + k;  // published after the deals (same copy stream)
    CUDA_TRY(cudaMemcpyAsync(st->d_words + 0, st->h_words + 0, 8, cudaMemcpyHostToDevice, st->cstream));
    CUDA_TRY(cudaStreamSynchronize(st->cstream));
    st->published += k;
  }
  if (accepted) *accepted = k;
  return stream_kernel(st);
}

int ddg_stream_poll(ddg_stream* st, uint8_t* rec28, int64_t max, int64_t* got) {
  if (got) *got = 0;
  if (!st) return fail(DDG_E_ARG, "null stream");
  if (max < 0 || (max > 0 && !rec28)) return fail(DDG_E_ARG, "bad poll arguments");
  const unsigned long long mask = (unsigned long long)st->slots - 1;
  int64_t k = 0;
  while (k < max) {
    volatile CompRec* r = st->h_comp + (st->consumed & mask);
    if (r->flag != (unsigned)(st->consumed + 1)) break;
    std::atomic_thread_fence(std::memory_order_acquire);
    const unsigned long long seq = r->seq;
    memcpy(rec28 + k * 28, &seq, 8);
    for (int b = 0; b < 20; b++) rec28[k * 28 + 8 + b] = r->tricks[b];
    st->slot_busy[seq & mask] = 0;
    st->consumed++;
    k++;
  }
  if (got) *got = k;
  if (st->published > st->consumed) {
    CUDA_TRY(cudaSetDevice(st->s->device));
    return stream_kernel(st);  // lanes that timed out come back for work still in flight
  }
  return DDG_OK;
}

int ddg_stream_close(ddg_stream* st, int drain, ddg_stats* stats) {
  if (!st) return fail(DDG_E_ARG, "null stream");
  if (stats) memset(stats, 0, sizeof(*stats));
  cudaSetDevice(st->s->device);
  if (!drain) *(volatile int*)st->s->h_stop = 1;  // blocks end at their next check
  st->h_words[3] = 1;  // closing: lanes end once every published deal is taken and done
  cudaError_t e = cudaMemcpyAsync(st->d_words + 3, st->h_words + 3, 8, cudaMemcpyHostToDevice, st->cstream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st->cstream);
  int rc = e == cudaSuccess ? DDG_OK : fail(DDG_E_CUDA, "stream close: %s", cudaGetErrorString(e));
  // The kernel ends when its lanes find nothing left; if it had timed out with work left,
  // one more launch finishes it.
  for (int round = 0; rc == DDG_OK && round < 2; round++) {
    e = cudaEventSynchronize(st->kdone);
    if (e != cudaSuccess) {
      rc = fail(DDG_E_CUDA, "stream kernel: %s", cudaGetErrorString(e));
      break;
    }
    st->launched = false;
    unsigned long long words[4];
    e = cudaMemcpy(words, st->d_words, sizeof(words), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      rc = fail(DDG_E_CUDA, "stream close: %s", cudaGetErrorString(e));
      break;
    }
    if (!drain || words[2] >= st->published) break;
    rc = stream_kernel(st);
  }
  if (rc == DDG_OK && stats) {
    unsigned long long c[CNT_WORDS];
    e = cudaMemcpy(c, st->s->counters, sizeof(c), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) {
      stats->nodes = c[CNT_NODES];
      stats->tt_probes = c[CNT_PROBES];
      stats->tt_hits = c[CNT_HITS];
      stats->tt_stores = c[CNT_STORES];
      stats->tt_bytes = c[CNT_TT_BYTES];
      for (int k = 0; k < 7; k++) stats->enter_exit[k] = c[CNT_EXIT + k];
      stats->jobs_done = (int64_t)c[CNT_JOBS_DONE];
      stats->iterations = c[CNT_ITERS];
      stats->lanes = st->s->lanes;
      stats->block = st->s->block;
      stats->grid = st->s->lanes / st->s->block;
      stats->tasks = (uint64_t)st->launches;
    }
    st->s->total_nodes += c[CNT_NODES];
  }
  stream_free(st);
  return rc;
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

// One job of one deal: strain `strain` for declarer `decl` (or all four, decl = -1), with
// seeds (stepping search) or a first target (binary search). out20 receives the deal's
// table row of that strain. The calls for one strain or one lead of the reference's API.
static int solve_one(ddg_solver* s, const uint64_t* hands4, int strain, int decl, const int8_t* seeds20,
                     int first_target, uint8_t* out20) {
  if (!s) return fail(DDG_E_ARG, "null solver");
  if (!hands4 || !out20) return fail(DDG_E_ARG, "null argument");
  if (strain < 0 || strain > 4) return fail(DDG_E_ARG, "strain %d is not 0..4", strain);
  if (s->streaming) return fail(DDG_E_STATE, "a stream is open on this solver");
  int rc = ddg_check_deal(hands4);
  if (rc) return rc;
  CUDA_TRY(cudaSetDevice(s->device));
  rc = ensure_staging(s, 1);
  if (rc) return rc;
  s->sliced = false;
  CUDA_TRY(cudaMemcpy(s->d_hands, hands4, 32, cudaMemcpyHostToDevice));
  if (seeds20) CUDA_TRY(cudaMemcpy(s->d_seeds, seeds20, 20, cudaMemcpyHostToDevice));
  BatchArgs a = make_args(s, s->d_hands, 1, seeds20 ? s->d_seeds : nullptr, s->d_out, nullptr);
  a.n_jobs = 1;
  a.one_job = 1;
  a.one_strain = strain;
  a.one_decl = decl;
  a.first_target = first_target;
  CUDA_TRY(cudaMemset(s->counters, 0, CNT_WORDS * 8));
  CUDA_TRY(cudaMemset(s->d_out, 0xFF, 20));
  if (s->tasks) CUDA_TRY(cudaMemset(s->tasks, 0, s->tasks_bytes));
  *(volatile int*)s->h_stop = 0;
  CUDA_TRY(cudaEventRecord(s->ev0, nullptr));
  int grid = 0;
  rc = launch_batch(s, a, 1, nullptr, &grid);
  if (rc) return rc;
  CUDA_TRY(cudaEventRecord(s->ev1, nullptr));
  rc = wait_launch(s);
  if (rc) return rc;
  unsigned long long c[CNT_WORDS];
  rc = read_stats(s, grid, nullptr, c);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpy(out20, s->d_out, 20, cudaMemcpyDeviceToHost));
  return DDG_OK;
}

int ddg_solve_strain(ddg_solver* s, const uint64_t* hands4, int strain, const int* ns4, int* out4) {
  if (!out4) return fail(DDG_E_ARG, "null output");
  int8_t seeds[20];
  for (int i = 0; i < 20; i++) seeds[i] = 7;
  if (ns4 && strain >= 0 && strain <= 4)
    for (int d = 0; d < 4; d++) seeds[strain * 4 + d] = (int8_t)ns4[d];
  uint8_t out[20];
  int rc = solve_one(s, hands4, strain, -1, ns4 ? seeds : nullptr, 0, out);
  if (rc) return rc;
  for (int d = 0; d < 4; d++) out4[d] = out[strain * 4 + d];
  return DDG_OK;
}

int ddg_ns_tricks(ddg_solver* s, const uint64_t* hands4, int strain, int leader, int guess, int stepping,
                  int* ns_out) {
  if (!ns_out) return fail(DDG_E_ARG, "null output");
  if (leader < 0 || leader > 3) return fail(DDG_E_ARG, "leader %d is not 0..3", leader);
  const int decl = (leader + 3) & 3;
  int8_t seeds[20];
  for (int i = 0; i < 20; i++) seeds[i] = (int8_t)(guess < -1 ? -1 : guess > 13 ? 13 : guess);
  uint8_t out[20];
  // The binary search clamps its first target to 1..13 (src/dd.h:881); the stepping
  // search clamps its seed to 0..tricks left (src/dd.h:903).
  const int first = guess < 1 ? 1 : guess > 13 ? 13 : guess;
  int rc = solve_one(s, hands4, strain, decl, stepping ? seeds : nullptr, stepping ? 0 : first, out);
  if (rc) return rc;
  const int v = out[strain * 4 + decl];
  *ns_out = (decl & 1) == 0 ? v : 13 - v;
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

void ddg_make_deals_mixed(uint64_t seed, int64_t first, int64_t n, int k_min, int k_max, double skew,
                          uint64_t* hands) {
  if (k_min < 1) k_min = 1;
  if (k_max > 13) k_max = 13;
  if (k_max < k_min) k_max = k_min;
  for (int64_t d = 0; d < n; d++) {
    uint64_t x = seed ^ (0x9E6C63D0676A9A99ull * (uint64_t)(first + d + 1));
    const int k = k_min + (int)(splitmix_next(x) % (uint64_t)(k_max - k_min + 1));
    uint64_t* h = hands + d * 4;
    h[0] = h[1] = h[2] = h[3] = 0;
    // A skewed deal: seat `lng` holds min(7..10, k) cards of suit `su`, seat `vd` none.
    const bool skewed = (double)(splitmix_next(x) >> 11) * (1.0 / 9007199254740992.0) < skew;
    int cards[52], m = 0;
    for (int i = 0; i < 52; i++) cards[i] = (i / 13) * 16 + i % 13;
    for (int i = 51; i > 0; i--) {  // shuffle all 52 first
      int j = (int)(splitmix_next(x) % (uint64_t)(i + 1));
      int t = cards[i];
      cards[i] = cards[j];
      cards[j] = t;
    }
    int cnt[4] = {0, 0, 0, 0};
    int su = -1, lng = -1, vd = -1;
    if (skewed) {
      su = (int)(splitmix_next(x) % 4);
      lng = (int)(splitmix_next(x) % 4);
      vd = (lng + 1 + (int)(splitmix_next(x) % 3)) % 4;
      int want = 7 + (int)(splitmix_next(x) % 4);
      if (want > k) want = k;
      for (int i = 0; i < 52 && cnt[lng] < want; i++)
        if (cards[i] >= 0 && (cards[i] >> 4) == su) {
          h[lng] |= 1ull << cards[i];
          cnt[lng]++;
          cards[i] = -1;
        }
    }
    // The void seat first (only cards of the other suits), then the rest in shuffled order,
    // round-robin over the seats that still need cards.
    if (skewed)
      for (int i = 0; i < 52 && cnt[vd] < k; i++)
        if (cards[i] >= 0 && (cards[i] >> 4) != su) {
          h[vd] |= 1ull << cards[i];
          cnt[vd]++;
          cards[i] = -1;
        }
    int seat = 0;
    for (int i = 0; i < 52; i++) {
      const int c = cards[i];
      if (c < 0) continue;
      for (int tries = 0; tries < 4; tries++, seat = (seat + 1) % 4) {
        if (cnt[seat] >= k) continue;
        if (seat == vd && (c >> 4) == su) continue;
        h[seat] |= 1ull << c;
        cnt[seat]++;
        seat = (seat + 1) % 4;
        break;
      }
      if (cnt[0] >= k && cnt[1] >= k && cnt[2] >= k && cnt[3] >= k) break;
    }
    (void)m;
  }
}

}  // extern "C"

#include "ddg_static.cuh"
#include "ddg_guide_api.cuh"
