// C ABI of the learned guide (include/ddg.h, ddg_guide_*): parameters, one training step
// (forward, loss, backward and Adam, all on the GPU in this file's kernels) and inference
// of NS seeds and root leads. Included at the end of ddg_api.cu.
#pragma once
#include "ddg_guide.cuh"

struct ddg_guide {
  int device = 0;
  int max_rows = 0;
  long long step = 0;
  float* master = nullptr;  // fp32 parameters (flat layout of guide_nn::N_PARAMS)
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  float* grad = nullptr;
  guide_nn::bf16 *w1 = nullptr, *w2 = nullptr, *w2t = nullptr, *w3 = nullptr, *w3t = nullptr;
  // workspace for max_rows rows
  guide_nn::bf16 *X = nullptr, *Xt = nullptr, *H1 = nullptr, *H1t = nullptr, *H2 = nullptr, *H2t = nullptr;
  guide_nn::bf16 *dO = nullptr, *dOt = nullptr, *dZ1 = nullptr, *dZ1t = nullptr, *dZ2 = nullptr, *dZ2t = nullptr;
  float *Z1 = nullptr, *Z2 = nullptr, *L = nullptr, *dW3full = nullptr;
  float* acc = nullptr;  // loss, hits, rows
  int64_t* rows_buf = nullptr;
  int* err = nullptr;
};

namespace guide_nn {

static bool g_attr_done[64];

static int set_gemm_attrs() {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && g_attr_done[dev]) return DDG_OK;
  CUDA_TRY(cudaFuncSetAttribute((const void*)gemm_tc<EPI_STORE>, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM));
  CUDA_TRY(cudaFuncSetAttribute((const void*)gemm_tc<EPI_BIAS_GELU>, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM));
  CUDA_TRY(cudaFuncSetAttribute((const void*)gemm_tc<EPI_BIAS>, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM));
  CUDA_TRY(cudaFuncSetAttribute((const void*)gemm_tc<EPI_GELU_BACK>, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM));
  if (dev >= 0 && dev < 64) g_attr_done[dev] = true;
  return DDG_OK;
}

// C = A . B^T with the fused epilogue; M % 128 == 0, N % 16 == 0, N <= 256, K % 64 == 0.
template <int EPI>
static int gemm(const GemmArgs& g, cudaStream_t st) {
  if (g.M % TILE_M || g.N % 16 || g.N > 256 || g.N < 16 || g.K % KCHUNK || g.lda % 8 || g.ldb % 8)
    return fail(DDG_E_ARG, "gemm shape %d x %d x %d", g.M, g.N, g.K);
  gemm_tc<EPI><<<g.M / TILE_M, 128, GEMM_SMEM, st>>>(g);
  CUDA_TRY(cudaGetLastError());
  return DDG_OK;
}

static GemmArgs gargs(const bf16* A, int lda, const bf16* B, int ldb, int M, int N, int K, int* err) {
  GemmArgs g;
  memset(&g, 0, sizeof(g));
  g.A = A;
  g.lda = lda;
  g.B = B;
  g.ldb = ldb;
  g.M = M;
  g.N = N;
  g.K = K;
  g.err = err;
  return g;
}

static int tr(const bf16* in, int ldi, int R, int C, bf16* out, int ldo, cudaStream_t st) {
  dim3 grid((C + 31) / 32, (R + 31) / 32), block(32, 8);
  transpose<<<grid, block, 0, st>>>(in, ldi, R, C, out, ldo);
  CUDA_TRY(cudaGetLastError());
  return DDG_OK;
}

static int refresh_bf16(ddg_guide* g, cudaStream_t st) {
  const int t = 256;
  to_bf16<<<(HID * IN_PAD + t - 1) / t, t, 0, st>>>(g->master + OFF_W1, HID, IN_PAD, g->w1, nullptr, 0);
  to_bf16<<<(HID * HID + t - 1) / t, t, 0, st>>>(g->master + OFF_W2, HID, HID, g->w2, g->w2t, HID);
  to_bf16<<<(OUT_PAD * HID + t - 1) / t, t, 0, st>>>(g->master + OFF_W3, OUT_PAD, HID, g->w3, g->w3t, DO_LD);
  CUDA_TRY(cudaGetLastError());
  return DDG_OK;
}

// Forward pass of rows 0..R-1 of X (R % 128 == 0): Z1/H1, Z2/H2, logits L.
static int forward(ddg_guide* g, int R, cudaStream_t st) {
  GemmArgs a = gargs(g->X, IN_PAD, g->w1, IN_PAD, R, HID, IN_PAD, g->err);
  a.C = g->Z1;
  a.ldc = HID;
  a.bias = g->master + OFF_B1;
  a.H = g->H1;
  a.ldh = HID;
  int rc = gemm<EPI_BIAS_GELU>(a, st);
  if (rc) return rc;
  GemmArgs b = gargs(g->H1, HID, g->w2, HID, R, HID, HID, g->err);
  b.C = g->Z2;
  b.ldc = HID;
  b.bias = g->master + OFF_B2;
  b.H = g->H2;
  b.ldh = HID;
  rc = gemm<EPI_BIAS_GELU>(b, st);
  if (rc) return rc;
  GemmArgs c = gargs(g->H2, HID, g->w3, HID, R, OUT_PAD, HID, g->err);
  c.C = g->L;
  c.ldc = OUT_PAD;
  c.bias = g->master + OFF_B3;
  return gemm<EPI_BIAS>(c, st);
}

static int check_err(ddg_guide* g) {
  int e = 0;
  CUDA_TRY(cudaMemcpy(&e, g->err, 4, cudaMemcpyDeviceToHost));
  if (e) return fail(DDG_E_TIMEOUT, "guide: a tensor-core product did not complete (bounded wait)");
  return DDG_OK;
}

}  // namespace guide_nn

extern "C" {

int64_t ddg_guide_param_count(void) { return guide_nn::N_PARAMS; }

void ddg_guide_destroy(ddg_guide* g) {
  if (!g) return;
  cudaSetDevice(g->device);
  void* bufs[] = {g->master, g->adam_m, g->adam_v, g->grad, g->w1, g->w2, g->w2t, g->w3, g->w3t, g->X, g->Xt,
                  g->H1, g->H1t, g->H2, g->H2t, g->dO, g->dOt, g->dZ1, g->dZ1t, g->dZ2, g->dZ2t, g->Z1, g->Z2,
                  g->L, g->dW3full, g->acc, g->rows_buf, g->err};
  for (void* b : bufs) cudaFree(b);
  delete g;
}

int ddg_guide_create(int device, int max_rows, const float* params, ddg_guide** out) {
  using namespace guide_nn;
  if (!out) return fail(DDG_E_ARG, "null output");
  *out = nullptr;
  if (max_rows <= 0 || max_rows % TILE_M || max_rows > (1 << 20))
    return fail(DDG_E_ARG, "max_rows %d is not a positive multiple of 128 (<= 1M)", max_rows);
  CUDA_TRY(cudaSetDevice(device));
  int rc = set_gemm_attrs();
  if (rc) return rc;
  ddg_guide* g = new ddg_guide();
  g->device = device;
  g->max_rows = max_rows;
  const size_t R = (size_t)max_rows, P = (size_t)N_PARAMS;
  cudaError_t e = cudaSuccess;
  auto A = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);
  };
  A((void**)&g->master, P * 4);
  A((void**)&g->adam_m, P * 4);
  A((void**)&g->adam_v, P * 4);
  A((void**)&g->grad, P * 4);
  A((void**)&g->w1, (size_t)HID * IN_PAD * 2);
  A((void**)&g->w2, (size_t)HID * HID * 2);
  A((void**)&g->w2t, (size_t)HID * HID * 2);
  A((void**)&g->w3, (size_t)OUT_PAD * HID * 2);
  A((void**)&g->w3t, (size_t)HID * DO_LD * 2);
  A((void**)&g->X, R * IN_PAD * 2);
  A((void**)&g->Xt, R * IN_PAD * 2);
  A((void**)&g->H1, R * HID * 2);
  A((void**)&g->H1t, R * HID * 2);
  A((void**)&g->H2, R * HID * 2);
  A((void**)&g->H2t, R * HID * 2);
  A((void**)&g->dO, R * DO_LD * 2);
  A((void**)&g->dOt, R * DO_LD * 2);
  A((void**)&g->dZ1, R * HID * 2);
  A((void**)&g->dZ1t, R * HID * 2);
  A((void**)&g->dZ2, R * HID * 2);
  A((void**)&g->dZ2t, R * HID * 2);
  A((void**)&g->Z1, R * HID * 4);
  A((void**)&g->Z2, R * HID * 4);
  A((void**)&g->L, R * OUT_PAD * 4);
  A((void**)&g->dW3full, (size_t)DO_LD * HID * 4);
  A((void**)&g->acc, 4 * 4);
  A((void**)&g->rows_buf, R * 8);
  A((void**)&g->err, 4);
  if (e == cudaSuccess && params) e = cudaMemcpy(g->master, params, P * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    ddg_guide_destroy(g);
    return fail(e == cudaErrorMemoryAllocation ? DDG_E_MEMORY : DDG_E_CUDA, "guide buffers: %s",
                cudaGetErrorString(e));
  }
  rc = refresh_bf16(g, nullptr);
  if (rc == DDG_OK && cudaDeviceSynchronize() != cudaSuccess) rc = fail(DDG_E_CUDA, "guide init");
  if (rc) {
    ddg_guide_destroy(g);
    return rc;
  }
  *out = g;
  return DDG_OK;
}

int ddg_guide_get_params(ddg_guide* g, float* params) {
  if (!g || !params) return fail(DDG_E_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(g->device));
  CUDA_TRY(cudaMemcpy(params, g->master, guide_nn::N_PARAMS * 4, cudaMemcpyDeviceToHost));
  return DDG_OK;
}

int ddg_guide_set_params(ddg_guide* g, const float* params) {
  if (!g || !params) return fail(DDG_E_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(g->device));
  CUDA_TRY(cudaMemcpy(g->master, params, guide_nn::N_PARAMS * 4, cudaMemcpyHostToDevice));
  int rc = guide_nn::refresh_bf16(g, nullptr);
  if (rc) return rc;
  CUDA_TRY(cudaDeviceSynchronize());
  return DDG_OK;
}

int ddg_guide_train_step(ddg_guide* g, const uint64_t* d_hands, const uint8_t* d_tricks20, const int8_t* d_best20,
                         const int64_t* rows_host, int n_rows, float lr, float* stats3, float* grad_host) {
  using namespace guide_nn;
  if (!g || !d_hands || !d_tricks20 || !d_best20 || !rows_host) return fail(DDG_E_ARG, "null argument");
  if (n_rows <= 0 || n_rows > g->max_rows) return fail(DDG_E_ARG, "%d rows (max %d)", n_rows, g->max_rows);
  CUDA_TRY(cudaSetDevice(g->device));
  const int R = (n_rows + TILE_M - 1) / TILE_M * TILE_M;  // padded rows carry no example
  std::vector<int64_t> rows(R, -1);
  for (int i = 0; i < n_rows; i++) rows[i] = rows_host[i];
  cudaStream_t st = nullptr;
  CUDA_TRY(cudaMemcpy(g->rows_buf, rows.data(), (size_t)R * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemsetAsync(g->acc, 0, 16, st));
  CUDA_TRY(cudaMemsetAsync(g->err, 0, 4, st));
  features<<<R, 64, 0, st>>>(d_hands, g->rows_buf, R, g->X);
  int rc = forward(g, R, st);
  if (rc) return rc;
  loss_grad<<<(R + 127) / 128, 128, 0, st>>>(g->L, d_hands, d_tricks20, d_best20, g->rows_buf, R, g->dO, g->acc);
  // Backward. Weight gradients: dW = dYᵀ . X as products over the batch (K = R).
  if ((rc = tr(g->dO, DO_LD, R, DO_LD, g->dOt, R, st)) || (rc = tr(g->H2, HID, R, HID, g->H2t, R, st)) ||
      (rc = tr(g->H1, HID, R, HID, g->H1t, R, st)) || (rc = tr(g->X, IN_PAD, R, IN_PAD, g->Xt, R, st)))
    return rc;
  GemmArgs w3 = gargs(g->dOt, R, g->H2t, R, DO_LD, HID, R, g->err);
  w3.C = g->dW3full;
  w3.ldc = HID;
  if ((rc = gemm<EPI_STORE>(w3, st))) return rc;
  CUDA_TRY(cudaMemcpyAsync(g->grad + OFF_W3, g->dW3full, (size_t)OUT_PAD * HID * 4, cudaMemcpyDeviceToDevice, st));
  colsum<<<1, 128, 0, st>>>(g->dO, DO_LD, R, OUT_PAD, g->grad + OFF_B3);
  GemmArgs h2 = gargs(g->dO, DO_LD, g->w3t, DO_LD, R, HID, DO_LD, g->err);  // dH2 = dO . W3
  h2.H = g->dZ2;
  h2.ldh = HID;
  h2.Z = g->Z2;
  h2.ldz = HID;
  if ((rc = gemm<EPI_GELU_BACK>(h2, st))) return rc;
  if ((rc = tr(g->dZ2, HID, R, HID, g->dZ2t, R, st))) return rc;
  GemmArgs w2 = gargs(g->dZ2t, R, g->H1t, R, HID, HID, R, g->err);
  w2.C = g->grad + OFF_W2;
  w2.ldc = HID;
  if ((rc = gemm<EPI_STORE>(w2, st))) return rc;
  colsum<<<2, 128, 0, st>>>(g->dZ2, HID, R, HID, g->grad + OFF_B2);
  GemmArgs h1 = gargs(g->dZ2, HID, g->w2t, HID, R, HID, HID, g->err);  // dH1 = dZ2 . W2
  h1.H = g->dZ1;
  h1.ldh = HID;
  h1.Z = g->Z1;
  h1.ldz = HID;
  if ((rc = gemm<EPI_GELU_BACK>(h1, st))) return rc;
  if ((rc = tr(g->dZ1, HID, R, HID, g->dZ1t, R, st))) return rc;
  GemmArgs w1 = gargs(g->dZ1t, R, g->Xt, R, HID, IN_PAD, R, g->err);
  w1.C = g->grad + OFF_W1;
  w1.ldc = IN_PAD;
  if ((rc = gemm<EPI_STORE>(w1, st))) return rc;
  colsum<<<2, 128, 0, st>>>(g->dZ1, HID, R, HID, g->grad + OFF_B1);
  CUDA_TRY(cudaGetLastError());
  if (grad_host) CUDA_TRY(cudaMemcpy(grad_host, g->grad, N_PARAMS * 4, cudaMemcpyDeviceToHost));
  if (lr > 0) {
    g->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)g->step), c2 = 1.f - powf(b2, (float)g->step);
    adam<<<(N_PARAMS + 255) / 256, 256, 0, st>>>(g->master, g->adam_m, g->adam_v, g->grad, N_PARAMS, lr, b1, b2,
                                                 1e-8f, c1, c2);
    if ((rc = refresh_bf16(g, st))) return rc;
  }
  CUDA_TRY(cudaDeviceSynchronize());
  if ((rc = check_err(g))) return rc;
  if (stats3) CUDA_TRY(cudaMemcpy(stats3, g->acc, 12, cudaMemcpyDeviceToHost));
  return DDG_OK;
}

int ddg_guide_predict(ddg_guide* g, const uint64_t* d_hands, int64_t n, int8_t* d_seed20, int8_t* d_hint20) {
  using namespace guide_nn;
  if (!g || (n > 0 && !d_hands)) return fail(DDG_E_ARG, "null argument");
  if (n < 0) return fail(DDG_E_ARG, "n < 0");
  CUDA_TRY(cudaSetDevice(g->device));
  int rc = guide_predict_on(g, d_hands, n, d_seed20, d_hint20, nullptr);
  if (rc) return rc;
  CUDA_TRY(cudaDeviceSynchronize());
  return check_err(g);
}

}  // extern "C"

// The inference of ddg_guide_predict on `stream`, waiting for that stream only: a guided
// stream calls it while its persistent solve kernel runs on another stream.
static int guide_predict_on(ddg_guide* g, const uint64_t* d_hands, int64_t n, int8_t* d_seed20, int8_t* d_hint20,
                            cudaStream_t stream) {
  using namespace guide_nn;
  CUDA_TRY(cudaMemsetAsync(g->err, 0, 4, stream));
  const int64_t total = n * 20;
  for (int64_t first = 0; first < total; first += g->max_rows) {
    const int rows = (int)std::min<int64_t>(g->max_rows, total - first);
    const int R = (rows + TILE_M - 1) / TILE_M * TILE_M;
    std::vector<int64_t> idx(R, -1);
    for (int i = 0; i < rows; i++) idx[i] = first + i;
    // from pageable memory: the call returns once the rows are staged, so idx may go
    CUDA_TRY(cudaMemcpyAsync(g->rows_buf, idx.data(), (size_t)R * 8, cudaMemcpyHostToDevice, stream));
    features<<<R, 64, 0, stream>>>(d_hands, g->rows_buf, R, g->X);
    int rc = forward(g, R, stream);
    if (rc) return rc;
    predict_out<<<(rows + 127) / 128, 128, 0, stream>>>(g->L, d_hands, first, rows, d_seed20, d_hint20);
    CUDA_TRY(cudaGetLastError());
  }
  if (stream) {
    CUDA_TRY(cudaStreamSynchronize(stream));
    return check_err(g);
  }
  return DDG_OK;
}

extern "C" {

}  // extern "C"
