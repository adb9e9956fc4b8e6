// The learned guide: a small MLP that seeds the trick search and orders the root lead.
//
//   input  217 = 52 cards x 4 owners (one-hot) + 5 strains + 4 leaders, padded to 256
//   hidden 256 GELU, 256 GELU (BF16 weights and activations, FP32 accumulate)
//   heads  14 NS-trick classes (softmax) + 52 lead-card scores (softmax over the leader's
//          cards), padded to 80 outputs
//
// Every matrix product, forward and backward, runs in gemm_tc: a tcgen05 (5th-generation
// tensor core) kernel for sm_100a. One CTA of 128 threads computes a 128 x N tile of
// C = A . B^T (A: M x K, B: N x K, both bf16 and K-contiguous in memory): the threads
// stage 64-wide K chunks of A and B in shared memory in the no-swizzle K-major core-matrix
// layout, one thread issues the tcgen05.mma instructions (accumulator in tensor memory),
// tcgen05.commit signals an mbarrier when they are done, and the epilogue reads the
// accumulator back with tcgen05.ld (bias, GELU or its derivative fused). The guide only
// changes where searches start and which lead is tried first; the exact searches decide
// every answer.
#pragma once
#include <cuda_bf16.h>

namespace guide_nn {

typedef __nv_bfloat16 bf16;

enum : int {
  IN = 217,
  IN_PAD = 256,
  HID = 256,
  OUT_T = 14,   // NS tricks 0..13
  OUT_M = 52,   // lead card (suit*13 + rank)
  OUT = OUT_T + OUT_M,
  OUT_PAD = 80,  // N of the last layer (a multiple of 16)
  DO_LD = 128,   // row length of dO: K of the dH2 = dO . W3 product (a multiple of 64)
  KCHUNK = 64,
  TILE_M = 128,
};

// Flat parameter layout (fp32): W1[256][256] b1[256] W2[256][256] b2[256] W3[80][256] b3[80].
constexpr int64_t OFF_W1 = 0, OFF_B1 = OFF_W1 + HID * IN_PAD, OFF_W2 = OFF_B1 + HID, OFF_B2 = OFF_W2 + HID * HID,
                  OFF_W3 = OFF_B2 + HID, OFF_B3 = OFF_W3 + OUT_PAD * HID, N_PARAMS = OFF_B3 + OUT_PAD;

enum Epi { EPI_STORE = 0, EPI_BIAS_GELU = 1, EPI_BIAS = 2, EPI_GELU_BACK = 3 };

struct GemmArgs {
  const bf16* A;
  int lda;
  const bf16* B;
  int ldb;
  int M, N, K;
  float* C;  // fp32 out: product (STORE), product + bias (BIAS), pre-activation (BIAS_GELU)
  int ldc;
  const float* bias;
  bf16* H;  // bf16 out: GELU(z) (BIAS_GELU) or dZ = product * GELU'(Z) (GELU_BACK)
  int ldh;
  const float* Z;  // GELU_BACK: the forward pre-activation
  int ldz;
  int* err;  // set when a bounded wait gives up
};

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor (tcgen05): start address, leading (K) and stride (M/N)
// byte offsets, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | (uint64_t)((lbo >> 4) & 0x3FFFu) << 16 |
         (uint64_t)((sbo >> 4) & 0x3FFFu) << 32 | (uint64_t)1 << 46;
}

// Instruction descriptor of kind::f16: D f32, A and B bf16, both K-major, M = 128, N.
__device__ __forceinline__ uint32_t instr_desc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TILE_M >> 4) << 24);
}

// Waits for the mbarrier phase with parity `parity`; false if it did not complete within
// the bound (the caller records an error and winds down).
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (int it = 0; it < (1 << 24); it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

template <int EPI>
__global__ void __launch_bounds__(128, 1) gemm_tc(GemmArgs g) {
  extern __shared__ __align__(128) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int N = g.N;
  unsigned char* sA = sm;                            // 128 x 64 bf16 = 16 KB
  unsigned char* sB = sm + TILE_M * KCHUNK * 2;      // N x 64 bf16 <= 32 KB
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + TILE_M * KCHUNK * 2 + 256 * KCHUNK * 2);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
  const uint32_t ncols = N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
  const uint32_t mbar_a = smem_u32(mbar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_a));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tslot;
  const int m0 = blockIdx.x * TILE_M;
  const uint32_t lbo_a = (TILE_M / 8) * 128, lbo_b = (uint32_t)(N / 8) * 128;
  const uint32_t idesc = instr_desc(N);
  const uint32_t sA_a = smem_u32(sA), sB_a = smem_u32(sB);
  bool ok = true;
  const int chunks = g.K / KCHUNK;
  for (int c = 0; c < chunks && ok; c++) {
    const int k0 = c * KCHUNK;
    // Stage A (128 rows) and B (N rows) x 64 K: 16-byte vectors into core matrices of
    // 8 rows x 16 bytes; core matrix (row/8, k/8) sits at ((k/8) * rows/8 + row/8) * 128.
    for (int v = tid; v < TILE_M * 8; v += 128) {
      const int row = v >> 3, kg = v & 7;
      const uint4 x = *reinterpret_cast<const uint4*>(g.A + (size_t)(m0 + row) * g.lda + k0 + kg * 8);
      *reinterpret_cast<uint4*>(sA + (kg * (TILE_M / 8) + (row >> 3)) * 128 + (row & 7) * 16) = x;
    }
    for (int v = tid; v < N * 8; v += 128) {
      const int row = v >> 3, kg = v & 7;
      const uint4 x = *reinterpret_cast<const uint4*>(g.B + (size_t)row * g.ldb + k0 + kg * 8);
      *reinterpret_cast<uint4*>(sB + (kg * (N / 8) + (row >> 3)) * 128 + (row & 7) * 16) = x;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the tensor cores
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      for (int j = 0; j < KCHUNK / 16; j++) {
        const uint64_t da = smem_desc(sA_a + 2 * j * lbo_a, lbo_a, 128);
        const uint64_t db = smem_desc(sB_a + 2 * j * lbo_b, lbo_b, 128);
        const uint32_t acc = (c > 0 || j > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
            ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar_a)
                   : "memory");
    }
    // The products have read this chunk (and written the accumulator) before it is reused.
    ok = __syncthreads_and(mbar_wait(mbar_a, (uint32_t)(c & 1)));
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (!ok) {  // give the products in flight one more bounded wait before TMEM is freed
      mbar_wait(mbar_a, (uint32_t)(c & 1));
      __syncthreads();
    }
  }
  if (!ok) {
    if (tid == 0) atomicExch(g.err, 1);
  } else {
    const int row = m0 + warp * 32 + lane;  // TMEM lane = row of the tile
    for (int c0 = 0; c0 < N; c0 += 16) {
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      for (int k = 0; k < 16; k++) {
        const int col = c0 + k;
        const float acc = __uint_as_float(r[k]);
        if (EPI == EPI_STORE) {
          g.C[(size_t)row * g.ldc + col] = acc;
        } else if (EPI == EPI_BIAS) {
          g.C[(size_t)row * g.ldc + col] = acc + g.bias[col];
        } else if (EPI == EPI_BIAS_GELU) {
          const float z = acc + g.bias[col];
          g.C[(size_t)row * g.ldc + col] = z;
          g.H[(size_t)row * g.ldh + col] = __float2bfloat16_rn(gelu(z));
        } else {
          g.H[(size_t)row * g.ldh + col] = __float2bfloat16_rn(acc * gelu_grad(g.Z[(size_t)row * g.ldz + col]));
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

constexpr int GEMM_SMEM = TILE_M * KCHUNK * 2 + 256 * KCHUNK * 2 + 16;

// ---- elementwise kernels ----------------------------------------------------------------

__device__ __forceinline__ int card_index(int bit) { return (bit >> 4) * 13 + (bit & 15); }
__device__ __forceinline__ int card_bit(int idx) { return (idx / 13) * 16 + idx % 13; }

// Example e of deal set d: deal e / 20, strain (e % 20) / 4, declarer e % 4, leader
// declarer + 1. Row r of X gets the features of example rows[r] (rows[r] < 0: zeros).
__global__ void features(const uint64_t* hands, const int64_t* rows, int n_rows, bf16* X) {
  const int r = blockIdx.x;
  const int64_t e = rows ? rows[r] : (int64_t)r;
  bf16* x = X + (size_t)r * IN_PAD;
  for (int c = threadIdx.x; c < IN_PAD; c += blockDim.x) x[c] = __float2bfloat16_rn(0.f);
  __syncthreads();
  if (e < 0 || r >= n_rows) return;
  const int64_t deal = e / 20;
  const int strain = (int)(e % 20) / 4, decl = (int)(e % 4), leader = (decl + 1) & 3;
  for (int seat = 0; seat < 4; seat++) {
    const uint64_t h = hands[deal * 4 + seat];
    for (int c = threadIdx.x; c < 52; c += blockDim.x)
      if ((h >> card_bit(c)) & 1) x[c * 4 + seat] = __float2bfloat16_rn(1.f);
  }
  if (threadIdx.x == 0) {
    x[208 + strain] = __float2bfloat16_rn(1.f);
    x[213 + leader] = __float2bfloat16_rn(1.f);
  }
}

// Softmax cross-entropy of both heads for row r; writes dO = (p - y) / B (bf16, row
// length DO_LD, zeros outside the heads) and adds the row's loss and hits to acc[0..2].
__global__ void loss_grad(const float* L, const uint64_t* hands, const uint8_t* tricks20, const int8_t* best20,
                          const int64_t* rows, int B, bf16* dO, float* acc) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= B) return;
  bf16* d = dO + (size_t)r * DO_LD;
  for (int c = 0; c < DO_LD; c++) d[c] = __float2bfloat16_rn(0.f);
  const int64_t e = rows[r];
  if (e < 0) return;
  const int64_t deal = e / 20;
  const int sd = (int)(e % 20), decl = sd % 4, leader = (decl + 1) & 3;
  const int t = tricks20[deal * 20 + sd];
  if (t > 13) return;
  const int ns = (decl & 1) == 0 ? t : 13 - t;
  const float* l = L + (size_t)r * OUT_PAD;
  const float inv = 1.0f / (float)B;
  float mx = -1e30f;
  for (int c = 0; c < OUT_T; c++) mx = fmaxf(mx, l[c]);
  float sum = 0.f;
  int arg = 0;
  for (int c = 0; c < OUT_T; c++) {
    sum += expf(l[c] - mx);
    if (l[c] > l[arg]) arg = c;
  }
  float loss = -(l[ns] - mx - logf(sum));
  for (int c = 0; c < OUT_T; c++) {
    const float p = expf(l[c] - mx) / sum;
    d[c] = __float2bfloat16_rn((p - (c == ns ? 1.f : 0.f)) * inv);
  }
  const int best = best20[deal * 20 + sd];
  const uint64_t own = hands[deal * 4 + leader];
  if (best >= 0 && ((own >> best) & 1)) {
    const int y = card_index(best);
    mx = -1e30f;
    for (int c = 0; c < OUT_M; c++)
      if ((own >> card_bit(c)) & 1) mx = fmaxf(mx, l[OUT_T + c]);
    sum = 0.f;
    for (int c = 0; c < OUT_M; c++)
      if ((own >> card_bit(c)) & 1) sum += expf(l[OUT_T + c] - mx);
    loss += -(l[OUT_T + y] - mx - logf(sum));
    for (int c = 0; c < OUT_M; c++)
      if ((own >> card_bit(c)) & 1) {
        const float p = expf(l[OUT_T + c] - mx) / sum;
        d[OUT_T + c] = __float2bfloat16_rn((p - (c == y ? 1.f : 0.f)) * inv);
      }
  }
  atomicAdd(acc + 0, loss * inv);
  atomicAdd(acc + 1, arg == ns ? 1.f : 0.f);
  atomicAdd(acc + 2, 1.f);
}

// out[c][r] = in[r][c] for an R x C bf16 matrix (row lengths ldi, ldo).
__global__ void transpose(const bf16* in, int ldi, int R, int C, bf16* out, int ldo) {
  __shared__ bf16 tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    tile[k][threadIdx.x] = (r < R && c < C) ? in[(size_t)r * ldi + c] : __float2bfloat16_rn(0.f);
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (c < C && r < R) out[(size_t)c * ldo + r] = tile[threadIdx.x][k];
  }
}

// out[c] = sum over rows of in[r][c] (the bias gradients), c < C.
__global__ void colsum(const bf16* in, int ld, int R, int C, float* out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  float s = 0.f;
  for (int r = 0; r < R; r++) s += __bfloat162float(in[(size_t)r * ld + c]);
  out[c] = s;
}

// Adam on the fp32 master parameters (p, m, v, gradient g, n values).
__global__ void adam(float* p, float* m, float* v, const float* g, int64_t n, float lr, float b1, float b2, float eps,
                     float c1, float c2) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  m[i] = b1 * m[i] + (1.f - b1) * gi;
  v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
  p[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}

// bf16 copies of the weights for the products: W (rows x cols, row-major) and, when out_t
// is given, its transpose (cols rows of length ldt; entries from column `rows` on keep
// their zeros).
__global__ void to_bf16(const float* w, int rows, int cols, bf16* out, bf16* out_t, int ldt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const int r = i / cols, c = i % cols;
  const bf16 x = __float2bfloat16_rn(w[i]);
  out[i] = x;
  if (out_t) out_t[(size_t)c * ldt + r] = x;
}

// Seeds and root leads from the logits: example e of row r gets the arg-max NS tricks
// (clamped to 0..13) and the leader's card with the highest lead score.
__global__ void predict_out(const float* L, const uint64_t* hands, int64_t first, int n, int8_t* seed20,
                            int8_t* hint20) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int64_t e = first + r;
  const int64_t deal = e / 20;
  const int sd = (int)(e % 20), decl = sd % 4, leader = (decl + 1) & 3;
  const float* l = L + (size_t)r * OUT_PAD;
  int arg = 0;
  for (int c = 1; c < OUT_T; c++)
    if (l[c] > l[arg]) arg = c;
  if (seed20) seed20[e] = (int8_t)arg;
  if (hint20) {
    const uint64_t own = hands[deal * 4 + leader];
    int best = -1;
    float bv = -1e30f;
    for (int c = 0; c < OUT_M; c++)
      if (((own >> card_bit(c)) & 1) && l[OUT_T + c] > bv) {
        bv = l[OUT_T + c];
        best = c;
      }
    hint20[e] = (int8_t)(best < 0 ? -1 : card_bit(best));
  }
}

}  // namespace guide_nn
