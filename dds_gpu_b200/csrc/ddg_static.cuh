// ddg_solve_static: the one entry point that allocates nothing (included at the end of
// ddg_api.cu, so it launches the same compiled batch kernel as the other calls).
//
// Its working memory is a file-scope device array, reserved when the module is loaded:
// STATIC_LANES lanes of 2^STATIC_TT_LOG2 TT buckets, their frame stacks, TT generations and
// the counter words (42.6 MB in all: 41.9 MB of TTs, 0.66 MB of stacks). A call only
// enqueues work: two memsets and one launch on the caller's stream; it never calls
// cudaMalloc, cudaFree or an allocating library. It runs the pooled solver's default
// schedule (at most 3 cheap stages per lane per pass).
//
// What must start at zero: the TT tag lines and the lanes' TT generations, which static
// device storage is when the module loads; later calls keep them (each job starts a new
// generation, so earlier entries are never taken for this job's). The job-queue head and
// the statistics words are zeroed by every call before its launch.
//
// The scratch is shared: calls must not overlap. Two calls in flight at once (on two
// streams, or from two threads) race on the same TTs and job counter and their results
// are undefined; the caller serialises them (one stream, or a synchronisation between).
#pragma once

namespace ddg_static {

enum : int { STATIC_LANES = 256, STATIC_TT_LOG2 = 9, STATIC_BLOCK = 256, STATIC_MAX_DEALS = 1 << 20 };

constexpr size_t round256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t TT_BYTES = (size_t)STATIC_LANES * (sizeof(ddg::TTBucket) << STATIC_TT_LOG2);
constexpr size_t STACK_BYTES = (size_t)STATIC_LANES * sizeof(ddg::Frame) * ddg::STACK_DEPTH;
constexpr size_t GEN_BYTES = (size_t)STATIC_LANES * 4;
constexpr size_t CNT_BYTES = (size_t)ddg::CNT_WORDS * 8;
constexpr size_t OFF_STACKS = round256(TT_BYTES);
constexpr size_t OFF_GEN = OFF_STACKS + round256(STACK_BYTES);
constexpr size_t OFF_CNT = OFF_GEN + round256(GEN_BYTES);
constexpr size_t SCRATCH_BYTES = OFF_CNT + round256(CNT_BYTES);
#ifndef DDG_TT_SIG
static_assert(SCRATCH_BYTES / 100000 == 426, "the scratch size stated in ddg.h is 42.6 MB");
#endif

static __device__ __align__(256) unsigned char g_scratch[SCRATCH_BYTES];

// Device address of the scratch, looked up once per device (cudaGetSymbolAddress); the
// kernel's shared-memory limit is raised at the same time.
struct DeviceSlot {
  std::once_flag once;
  unsigned char* base = nullptr;
  cudaError_t err = cudaSuccess;
};
static DeviceSlot g_slots[64];

}  // namespace ddg_static

extern "C" int ddg_solve_static(const uint64_t* d_hands, int64_t n, uint8_t* d_out20, void* stream_v) {
  using namespace ddg_static;
  if (n < 0 || (n > 0 && (!d_hands || !d_out20))) return fail(DDG_E_ARG, "bad arguments");
  if (n > STATIC_MAX_DEALS)
    return fail(DDG_E_ARG, "%lld deals: ddg_solve_static takes at most %d per call", (long long)n, STATIC_MAX_DEALS);
  if ((reinterpret_cast<uintptr_t>(d_hands) & 15) != 0) return fail(DDG_E_ARG, "hands not 16-byte aligned");
  if (n == 0) return DDG_OK;
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(DDG_E_ARG, "device %d", dev);
  DeviceSlot& slot = g_slots[dev];
  std::call_once(slot.once, [&slot] {
    void* p = nullptr;
    slot.err = cudaGetSymbolAddress(&p, g_scratch);
    if (slot.err == cudaSuccess)
      slot.err = cudaFuncSetAttribute((const void*)ddg::batch_kernel<STATIC_BLOCK, 2>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sizeof(ddg::BlockShared<STATIC_BLOCK>));
    slot.base = static_cast<unsigned char*>(p);
  });
  if (slot.err != cudaSuccess) return fail(DDG_E_CUDA, "static scratch: %s", cudaGetErrorString(slot.err));
  cudaStream_t stream = (cudaStream_t)stream_v;
  ddg::BatchArgs a;
  memset(&a, 0, sizeof(a));
  a.hands = d_hands;
  a.n_jobs = (long long)n * 5;
  a.jpd = 5;
  a.mode = ddg::MODE_BISECT;
  a.out20 = d_out20;
  a.counters = reinterpret_cast<unsigned long long*>(slot.base + OFF_CNT);
  a.next_job = a.counters + ddg::CNT_NEXT_JOB;
  a.tt = reinterpret_cast<ddg::TTBucket*>(slot.base);
  a.stacks = reinterpret_cast<ddg::Frame*>(slot.base + OFF_STACKS);
  a.lane_gen = reinterpret_cast<ddg::u32*>(slot.base + OFF_GEN);
  a.tt_log2 = STATIC_TT_LOG2;
  a.free_below = 96;
  a.free_steps = 256;
  a.free_pack = 0;
  a.cheap_limit = 3;  // the pooled solver's default schedule (ddg_config.cheap_limit = 0)
  CUDA_TRY(cudaMemsetAsync(a.counters, 0, CNT_BYTES, stream));
  CUDA_TRY(cudaMemsetAsync(d_out20, 0xFF, (size_t)n * 20, stream));
  void* params[] = {&a};
  CUDA_TRY(cudaLaunchKernel((const void*)ddg::batch_kernel<STATIC_BLOCK, 2>, dim3(STATIC_LANES / STATIC_BLOCK),
                            dim3(STATIC_BLOCK), params, sizeof(ddg::BlockShared<STATIC_BLOCK>), stream));
  return DDG_OK;
}
