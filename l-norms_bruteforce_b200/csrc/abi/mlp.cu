// The proposal network: 44 -> 256 -> 256 -> 44, ReLU, bf16 operands with
// fp32 accumulation on the tensor cores (mlp_tc.cuh), trained with Adam on
// fp32 master weights.  Every GEMM of the forward and backward passes is
// C = A * B^T with both operands K-major; transposed copies of activations,
// gradients and weights are written by the kernels that produce them.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "../host/ld_internal.h"
#include "../kernels/mlp_tc.cuh"
#include "device_guard.h"

namespace {

using bf16 = __nv_bfloat16;
constexpr int kIn = 44, kInP = 64, kHid = 256, kOut = 44, kOutP = 64, kOutGP = 128;

#define MLP_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return ld_fail(LD_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

template <int BN>
size_t gemm_smem() {
  // Each CTA holds BN of the SM's 512 TMEM columns; the shared-memory request
  // is raised so that no more CTAs share an SM than TMEM can hold at once
  // (233472 bytes of shared memory per SM, 1 KB reserved per CTA).
  const size_t tiles = 2 * ((size_t)ld::mlp::kTileM * ld::mlp::kTileK * 2 + (size_t)BN * ld::mlp::kTileK * 2);
  const size_t cap = 233472 / (512 / BN + 1) + 1024;
  return tiles > cap ? tiles : cap;
}

// Shared-memory limits of the three GEMM instances; called before any
// launch on the current device (and before any stream capture).
cudaError_t gemm_init() {
  cudaError_t e = cudaFuncSetAttribute(ld::mlp::tc_gemm_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)gemm_smem<64>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ld::mlp::tc_gemm_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)gemm_smem<128>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ld::mlp::tc_gemm_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)gemm_smem<256>());
  return e;
}

template <int BN>
cudaError_t launch_gemm(const ld::mlp::GemmArgs& g, cudaStream_t s) {
  dim3 grid(g.M / ld::mlp::kTileM, g.N / BN);
  ld::mlp::tc_gemm_kernel<BN><<<grid, 128, gemm_smem<BN>(), s>>>(g);
  return cudaGetLastError();
}

cudaError_t gemm(const bf16* A, const bf16* B, int M, int N, int K, float* C, bf16* H, bf16* HT,
                 const float* bias, int relu, int* err, cudaStream_t s) {
  ld::mlp::GemmArgs g{A, B, M, N, K, C, H, HT, bias, relu, err};
  // these GEMMs are small: prefer the tile width that gives the most CTAs
  // while a wider tile still fills the 148 SMs
  const int tiles_m = M / ld::mlp::kTileM;
  if (N % 256 == 0 && tiles_m * (N / 256) >= 148) return launch_gemm<256>(g, s);
  if (N % 128 == 0 && tiles_m * (N / 128) >= 148) return launch_gemm<128>(g, s);
  return launch_gemm<64>(g, s);
}

int blocks_for(int n, int t = 256) { return (n + t - 1) / t; }

}  // namespace

struct ld_mlp {
  int device = 0, batch = 0;
  float skip = 0.f;
  cudaStream_t s = nullptr;
  void* mem = nullptr;
  // fp32 master parameters (padded shapes), gradients, Adam moments
  float *W1, *b1, *W2, *b2, *W3, *b3;
  float *gW1, *gb1, *gW2, *gb2, *gW3, *gb3;
  float *m[6], *v[6];
  // bf16 operands
  bf16 *W1b, *W2b, *W2T, *W3b, *W3T;
  bf16 *Xb, *XT, *H1, *H1T, *H2, *H2T, *dZ3, *dZ3T, *dZ2, *dZ2T, *dZ1T;
  float *Xf, *Z3, *Tt, *Mk, *dH2, *dH1, *loss, *hp;
  int* err;
  int step = 0;
  // pinned staging: inputs (x, targets, mask, step parameters) and results
  // (logits, loss, error flag); the graphs copy from and to these
  void* hmem = nullptr;
  float *hX, *hT, *hM, *hHp, *hZ, *hLoss;
  int* hErr;
  // captured CUDA graphs: one training step, one forward pass
  cudaGraphExec_t train_exec = nullptr, fwd_exec = nullptr;
};

namespace {

// parameter shapes (rows, cols) in the padded device layout and in the flat
// host layout used by get/set (unpadded)
struct PShape { int rows, cols, hrows, hcols; };
const PShape kShapes[6] = {{kHid, kInP, kHid, kIn}, {1, kHid, 1, kHid},   {kHid, kHid, kHid, kHid},
                           {1, kHid, 1, kHid},      {kOutP, kHid, kOut, kHid}, {1, kOutP, 1, kOut}};

float** params_of(ld_mlp* n, int i) {
  float** arr[6] = {&n->W1, &n->b1, &n->W2, &n->b2, &n->W3, &n->b3};
  return arr[i];
}
float** grads_of(ld_mlp* n, int i) {
  float** arr[6] = {&n->gW1, &n->gb1, &n->gW2, &n->gb2, &n->gW3, &n->gb3};
  return arr[i];
}

size_t host_param_count() {
  size_t c = 0;
  for (const auto& s : kShapes) c += (size_t)s.hrows * s.hcols;
  return c;
}

// refresh the bf16 copies of the weights from the fp32 masters
cudaError_t refresh_bf16(ld_mlp* n) {
  ld::mlp::to_bf16_kernel<<<blocks_for(kHid * kInP), 256, 0, n->s>>>(n->W1, kHid, kInP, n->W1b, nullptr);
  ld::mlp::to_bf16_kernel<<<blocks_for(kHid * kHid), 256, 0, n->s>>>(n->W2, kHid, kHid, n->W2b, n->W2T);
  ld::mlp::to_bf16_kernel<<<blocks_for(kOutP * kHid), 256, 0, n->s>>>(n->W3, kOutP, kHid, n->W3b, n->W3T);
  return cudaGetLastError();
}

// Host staging of one batch: rows of x (44 features) and, for training, of
// targets and mask, zero-padded to the device layout (batch x 64).  Returns
// 1 / (number of unmasked targets), or 0 when there are none.
float stage_batch(ld_mlp* n, const float* x, const float* t, const float* mask, int rows) {
  memset(n->hX, 0, sizeof(float) * (size_t)n->batch * kInP);
  for (int r = 0; r < rows; ++r) memcpy(n->hX + (size_t)r * kInP, x + (size_t)r * kIn, sizeof(float) * kIn);
  if (!t) return 0.f;
  memset(n->hT, 0, sizeof(float) * (size_t)n->batch * kOutP);
  memset(n->hM, 0, sizeof(float) * (size_t)n->batch * kOutP);
  double cnt = 0;
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < kOut; ++c) {
      n->hT[(size_t)r * kOutP + c] = t[(size_t)r * kOut + c];
      n->hM[(size_t)r * kOutP + c] = mask[(size_t)r * kOut + c];
      cnt += mask[(size_t)r * kOut + c];
    }
  return cnt > 0 ? (float)(1.0 / cnt) : 0.f;
}

// the staged inputs to the device, x to bf16 (and transposed)
cudaError_t enqueue_upload(ld_mlp* n, bool targets) {
  const size_t bx = sizeof(float) * (size_t)n->batch * kInP, bt = sizeof(float) * (size_t)n->batch * kOutP;
  cudaError_t e = cudaMemcpyAsync(n->Xf, n->hX, bx, cudaMemcpyHostToDevice, n->s);
  if (e == cudaSuccess && targets) e = cudaMemcpyAsync(n->Tt, n->hT, bt, cudaMemcpyHostToDevice, n->s);
  if (e == cudaSuccess && targets) e = cudaMemcpyAsync(n->Mk, n->hM, bt, cudaMemcpyHostToDevice, n->s);
  if (e == cudaSuccess && targets)
    e = cudaMemcpyAsync(n->hp, n->hHp, sizeof(float) * ld::mlp::kHpWords, cudaMemcpyHostToDevice, n->s);
  if (e != cudaSuccess) return e;
  ld::mlp::to_bf16_kernel<<<blocks_for(n->batch * kInP), 256, 0, n->s>>>(n->Xf, n->batch, kInP, n->Xb, n->XT);
  return cudaGetLastError();
}

cudaError_t enqueue_forward(ld_mlp* n) {
  const int B = n->batch;
  cudaError_t e = gemm(n->Xb, n->W1b, B, kHid, kInP, nullptr, n->H1, n->H1T, n->b1, 1, n->err, n->s);
  if (e == cudaSuccess) e = gemm(n->H1, n->W2b, B, kHid, kHid, nullptr, n->H2, n->H2T, n->b2, 1, n->err, n->s);
  if (e == cudaSuccess) e = gemm(n->H2, n->W3b, B, kOutP, kHid, n->Z3, nullptr, nullptr, n->b3, 0, n->err, n->s);
  return e;
}

cudaError_t enqueue_backward(ld_mlp* n) {
  const int B = n->batch;
  cudaError_t e = cudaMemsetAsync(n->loss, 0, sizeof(float), n->s);
  if (e != cudaSuccess) return e;
  // Xf and Z3 share the padded 64-column layout, so the residual input of
  // output column c is input column c
  static_assert(kInP == kOutP, "residual path needs equal padded widths");
  ld::mlp::bce_grad_kernel<<<blocks_for(B * kOutP), 256, 0, n->s>>>(n->Z3, n->Tt, n->Mk, B, kOutP, n->hp,
                                                                     n->skip != 0.f ? n->Xf : nullptr, n->skip,
                                                                     n->dZ3, n->dZ3T, n->loss);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  // W3: [kOutGP x B] x [kHid x B]^T (rows kOutP.. of dZ3T are zero)
  if ((e = gemm(n->dZ3T, n->H2T, kOutGP, kHid, B, n->gW3, nullptr, nullptr, nullptr, 0, n->err, n->s)) != cudaSuccess) return e;
  if ((e = gemm(n->dZ3, n->W3T, B, kHid, kOutP, n->dH2, nullptr, nullptr, nullptr, 0, n->err, n->s)) != cudaSuccess) return e;
  ld::mlp::relu_grad_kernel<<<blocks_for(B * kHid), 256, 0, n->s>>>(n->dH2, n->H2, B, kHid, n->dZ2, n->dZ2T);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = gemm(n->dZ2T, n->H1T, kHid, kHid, B, n->gW2, nullptr, nullptr, nullptr, 0, n->err, n->s)) != cudaSuccess) return e;
  if ((e = gemm(n->dZ2, n->W2T, B, kHid, kHid, n->dH1, nullptr, nullptr, nullptr, 0, n->err, n->s)) != cudaSuccess) return e;
  ld::mlp::relu_grad_kernel<<<blocks_for(B * kHid), 256, 0, n->s>>>(n->dH1, n->H1, B, kHid, nullptr, n->dZ1T);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = gemm(n->dZ1T, n->XT, kHid, kInP, B, n->gW1, nullptr, nullptr, nullptr, 0, n->err, n->s)) != cudaSuccess) return e;
  ld::mlp::bias_grad_kernel<<<kHid / 4, 128, 0, n->s>>>(n->dZ1T, kHid, B, n->gb1);
  ld::mlp::bias_grad_kernel<<<kHid / 4, 128, 0, n->s>>>(n->dZ2T, kHid, B, n->gb2);
  ld::mlp::bias_grad_kernel<<<kOutP / 4, 128, 0, n->s>>>(n->dZ3T, kOutP, B, n->gb3);
  return cudaGetLastError();
}

cudaError_t enqueue_adam(ld_mlp* n) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int i = 0; i < 6; ++i) {
    const PShape& sh = kShapes[i];
    bf16* wb = i == 0 ? n->W1b : i == 2 ? n->W2b : i == 4 ? n->W3b : nullptr;
    bf16* wbT = i == 2 ? n->W2T : i == 4 ? n->W3T : nullptr;
    ld::mlp::adam_kernel<<<blocks_for(sh.rows * sh.cols), 256, 0, n->s>>>(
        *params_of(n, i), *grads_of(n, i), n->m[i], n->v[i], sh.rows, sh.cols, n->hp, b1, b2, eps, wb, wbT);
  }
  return cudaGetLastError();
}

// loss and error flag (and, for a forward pass, the logits) back to staging
cudaError_t enqueue_results(ld_mlp* n, bool logits) {
  cudaError_t e = cudaMemcpyAsync(n->hLoss, n->loss, sizeof(float), cudaMemcpyDeviceToHost, n->s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(n->hErr, n->err, sizeof(int), cudaMemcpyDeviceToHost, n->s);
  if (e == cudaSuccess && logits)
    e = cudaMemcpyAsync(n->hZ, n->Z3, sizeof(float) * (size_t)n->batch * kOutP, cudaMemcpyDeviceToHost, n->s);
  return e;
}

// Capture `body` on the network's stream into an executable graph.
template <typename F>
ld_status capture(ld_mlp* n, F body, cudaGraphExec_t* out) {
  cudaGraph_t g = nullptr;
  MLP_CUDA(cudaStreamBeginCapture(n->s, cudaStreamCaptureModeThreadLocal));
  const cudaError_t e = body();
  const cudaError_t e2 = cudaStreamEndCapture(n->s, &g);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return ld_fail(LD_ERR_CUDA, "network graph capture failed: %s",
                   cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  const cudaError_t e3 = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e3 != cudaSuccess) return ld_fail(LD_ERR_CUDA, "network graph: %s", cudaGetErrorString(e3));
  return LD_OK;
}

// wait for the stream; report (and clear) a GEMM whose bounded wait ran out
ld_status finish(ld_mlp* n) {
  MLP_CUDA(cudaStreamSynchronize(n->s));
  if (*n->hErr) {
    const int e = *n->hErr;
    *n->hErr = 0;
    cudaMemsetAsync(n->err, 0, sizeof(int), n->s);
    cudaStreamSynchronize(n->s);
    return ld_fail(LD_ERR_TIMEOUT, "tensor-core GEMM wait ran out (code %d)", e);
  }
  return LD_OK;
}

}  // namespace

extern "C" ld_status ld_mlp_create(int32_t batch, uint64_t seed, float skip, int32_t device, ld_mlp** out) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
  if (!out || batch < 128 || batch % 128) return ld_fail(LD_ERR_ARG, "batch must be a positive multiple of 128");
  if (cudaSetDevice(device) != cudaSuccess) return ld_fail(LD_ERR_NODEV, "no device %d", device);
  ld_mlp* n = new ld_mlp();
  n->device = device;
  n->batch = batch;
  n->skip = skip;
  const int B = batch;
  // one allocation, carved in 256-byte aligned pieces
  struct Piece { void** p; size_t bytes; };
  std::vector<Piece> pieces;
  auto f32 = [&](float** p, size_t count) { pieces.push_back({(void**)p, count * 4}); };
  auto b16 = [&](bf16** p, size_t count) { pieces.push_back({(void**)p, count * 2}); };
  for (int i = 0; i < 6; ++i) {
    const size_t c = (size_t)kShapes[i].rows * kShapes[i].cols;
    f32(params_of(n, i), c);
    f32(grads_of(n, i), i == 4 ? (size_t)kOutGP * kHid : c);
    f32(&n->m[i], c);
    f32(&n->v[i], c);
  }
  b16(&n->W1b, (size_t)kHid * kInP); b16(&n->W2b, (size_t)kHid * kHid); b16(&n->W2T, (size_t)kHid * kHid);
  b16(&n->W3b, (size_t)kOutP * kHid); b16(&n->W3T, (size_t)kHid * kOutP);
  b16(&n->Xb, (size_t)B * kInP); b16(&n->XT, (size_t)kInP * B);
  b16(&n->H1, (size_t)B * kHid); b16(&n->H1T, (size_t)kHid * B);
  b16(&n->H2, (size_t)B * kHid); b16(&n->H2T, (size_t)kHid * B);
  b16(&n->dZ3, (size_t)B * kOutP); b16(&n->dZ3T, (size_t)kOutGP * B);
  b16(&n->dZ2, (size_t)B * kHid); b16(&n->dZ2T, (size_t)kHid * B); b16(&n->dZ1T, (size_t)kHid * B);
  f32(&n->Xf, (size_t)B * kInP); f32(&n->Z3, (size_t)B * kOutP); f32(&n->Tt, (size_t)B * kOutP);
  f32(&n->Mk, (size_t)B * kOutP); f32(&n->dH2, (size_t)B * kHid); f32(&n->dH1, (size_t)B * kHid);
  f32(&n->loss, 1);
  f32(&n->hp, ld::mlp::kHpWords);
  pieces.push_back({(void**)&n->err, 4});
  size_t total = 0;
  for (auto& pc : pieces) total += (pc.bytes + 255) & ~(size_t)255;
  if (cudaMalloc(&n->mem, total) != cudaSuccess || cudaStreamCreateWithFlags(&n->s, cudaStreamNonBlocking) != cudaSuccess) {
    if (n->mem) cudaFree(n->mem);
    delete n;
    return ld_fail(LD_ERR_CUDA, "network allocation of %zu bytes failed", total);
  }
  cudaMemset(n->mem, 0, total);
  size_t off = 0;
  for (auto& pc : pieces) { *pc.p = (char*)n->mem + off; off += (pc.bytes + 255) & ~(size_t)255; }
  // He-uniform initialisation of the real (unpadded) weights, zero biases
  std::mt19937_64 rng(seed);
  for (int i = 0; i < 6; i += 2) {
    const PShape& sh = kShapes[i];
    std::vector<float> w((size_t)sh.rows * sh.cols, 0.f);
    const float lim = std::sqrt(6.f / (float)sh.hcols);
    std::uniform_real_distribution<float> U(-lim, lim);
    for (int r = 0; r < sh.hrows; ++r)
      for (int c = 0; c < sh.hcols; ++c) w[(size_t)r * sh.cols + c] = U(rng);
    cudaMemcpy(*params_of(n, i), w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice);
  }
  if (refresh_bf16(n) != cudaSuccess || cudaStreamSynchronize(n->s) != cudaSuccess || gemm_init() != cudaSuccess) {
    ld_mlp_destroy(n);
    return ld_fail(LD_ERR_CUDA, "network initialisation failed");
  }
  // pinned staging: x, targets, mask (batch x 64 each), logits (batch x 64),
  // step parameters, loss, error flag
  const size_t slab = sizeof(float) * (size_t)B * 64;
  if (cudaMallocHost(&n->hmem, 4 * slab + 256) != cudaSuccess) {
    ld_mlp_destroy(n);
    return ld_fail(LD_ERR_CUDA, "pinned staging allocation failed");
  }
  char* h = (char*)n->hmem;
  n->hX = (float*)h; n->hT = (float*)(h + slab); n->hM = (float*)(h + 2 * slab); n->hZ = (float*)(h + 3 * slab);
  n->hHp = (float*)(h + 4 * slab); n->hLoss = (float*)(h + 4 * slab + 64); n->hErr = (int*)(h + 4 * slab + 128);
  memset(n->hmem, 0, 4 * slab + 256);
  // one training step and one forward pass as CUDA graphs over fixed buffers
  ld_status st = capture(n, [&] {
    cudaError_t e = enqueue_upload(n, true);
    if (e == cudaSuccess) e = enqueue_forward(n);
    if (e == cudaSuccess) e = enqueue_backward(n);
    if (e == cudaSuccess) e = enqueue_adam(n);
    if (e == cudaSuccess) e = enqueue_results(n, false);
    return e;
  }, &n->train_exec);
  if (st == LD_OK)
    st = capture(n, [&] {
      cudaError_t e = enqueue_upload(n, false);
      if (e == cudaSuccess) e = enqueue_forward(n);
      if (e == cudaSuccess) e = enqueue_results(n, true);
      return e;
    }, &n->fwd_exec);
  if (st != LD_OK) {
    ld_mlp_destroy(n);
    return st;
  }
  *out = n;
  return LD_OK;
}

extern "C" void ld_mlp_destroy(ld_mlp* n) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
  if (!n) return;
  cudaSetDevice(n->device);
  if (n->s) cudaStreamSynchronize(n->s);
  if (n->train_exec) cudaGraphExecDestroy(n->train_exec);
  if (n->fwd_exec) cudaGraphExecDestroy(n->fwd_exec);
  if (n->s) cudaStreamDestroy(n->s);
  if (n->mem) cudaFree(n->mem);
  if (n->hmem) cudaFreeHost(n->hmem);
  delete n;
}

extern "C" int64_t ld_mlp_param_count(void) { return (int64_t)host_param_count(); }

extern "C" ld_status ld_mlp_get_params(ld_mlp* n, float* params) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
  if (!n || !params) return ld_fail(LD_ERR_ARG, "null argument");
  MLP_CUDA(cudaSetDevice(n->device));
  MLP_CUDA(cudaStreamSynchronize(n->s));
  float* dst = params;
  for (int i = 0; i < 6; ++i) {
    const PShape& sh = kShapes[i];
    std::vector<float> w((size_t)sh.rows * sh.cols);
    MLP_CUDA(cudaMemcpy(w.data(), *params_of(n, i), sizeof(float) * w.size(), cudaMemcpyDeviceToHost));
    for (int r = 0; r < sh.hrows; ++r)
      for (int c = 0; c < sh.hcols; ++c) *dst++ = w[(size_t)r * sh.cols + c];
  }
  return LD_OK;
}

extern "C" ld_status ld_mlp_set_params(ld_mlp* n, const float* params) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
  if (!n || !params) return ld_fail(LD_ERR_ARG, "null argument");
  MLP_CUDA(cudaSetDevice(n->device));
  const float* src = params;
  for (int i = 0; i < 6; ++i) {
    const PShape& sh = kShapes[i];
    std::vector<float> w((size_t)sh.rows * sh.cols, 0.f);
    for (int r = 0; r < sh.hrows; ++r)
      for (int c = 0; c < sh.hcols; ++c) w[(size_t)r * sh.cols + c] = *src++;
    MLP_CUDA(cudaMemcpy(*params_of(n, i), w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice));
  }
  MLP_CUDA(refresh_bf16(n));
  MLP_CUDA(cudaStreamSynchronize(n->s));
  return LD_OK;
}

extern "C" ld_status ld_mlp_forward(ld_mlp* n, const float* x, int32_t rows, float* logits) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
  if (!n || !x || !logits || rows < 1) return ld_fail(LD_ERR_ARG, "bad arguments");
  MLP_CUDA(cudaSetDevice(n->device));
  for (int r0 = 0; r0 < rows; r0 += n->batch) {
    const int cnt = std::min(n->batch, rows - r0);
    stage_batch(n, x + (size_t)r0 * kIn, nullptr, nullptr, cnt);
    MLP_CUDA(cudaGraphLaunch(n->fwd_exec, n->s));
    ld_status st = finish(n);
    if (st != LD_OK) return st;
    for (int r = 0; r < cnt; ++r)
      for (int c = 0; c < kOut; ++c)
        logits[(size_t)(r0 + r) * kOut + c] = n->hZ[(size_t)r * kOutP + c] + n->skip * x[(size_t)(r0 + r) * kIn + c];
  }
  return LD_OK;
}

// gradients of the mean masked BCE loss (flat host layout), no update
extern "C" ld_status ld_mlp_gradients(ld_mlp* n, const float* x, const float* t, const float* mask, int32_t rows,
                                      float* grads, float* loss) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
  if (!n || !x || !t || !mask || rows < 1 || rows > n->batch) return ld_fail(LD_ERR_ARG, "bad arguments");
  MLP_CUDA(cudaSetDevice(n->device));
  n->hHp[ld::mlp::kHpInvCount] = stage_batch(n, x, t, mask, rows);
  MLP_CUDA(enqueue_upload(n, true));
  MLP_CUDA(enqueue_forward(n));
  MLP_CUDA(enqueue_backward(n));
  MLP_CUDA(enqueue_results(n, false));
  ld_status st = finish(n);
  if (st != LD_OK) return st;
  if (loss) *loss = *n->hLoss;
  if (grads) {
    float* dst = grads;
    for (int i = 0; i < 6; ++i) {
      const PShape& sh = kShapes[i];
      const int drows = i == 4 ? kOutGP : sh.rows;
      std::vector<float> g((size_t)drows * sh.cols);
      MLP_CUDA(cudaMemcpy(g.data(), *grads_of(n, i), sizeof(float) * g.size(), cudaMemcpyDeviceToHost));
      for (int r = 0; r < sh.hrows; ++r)
        for (int c = 0; c < sh.hcols; ++c) *dst++ = g[(size_t)r * sh.cols + c];
    }
  }
  return LD_OK;
}

// One Adam step: a single launch of the captured training graph.
extern "C" ld_status ld_mlp_train_step(ld_mlp* n, const float* x, const float* t, const float* mask, int32_t rows,
                                       float lr, float* loss) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
  if (!n || !x || !t || !mask || rows < 1 || rows > n->batch) return ld_fail(LD_ERR_ARG, "bad arguments");
  MLP_CUDA(cudaSetDevice(n->device));
  n->step += 1;
  n->hHp[ld::mlp::kHpInvCount] = stage_batch(n, x, t, mask, rows);
  n->hHp[ld::mlp::kHpLr] = lr;
  n->hHp[ld::mlp::kHpC1] = 1.f - std::pow(0.9f, (float)n->step);
  n->hHp[ld::mlp::kHpC2] = 1.f - std::pow(0.999f, (float)n->step);
  MLP_CUDA(cudaGraphLaunch(n->train_exec, n->s));
  ld_status st = finish(n);
  if (st != LD_OK) return st;
  if (loss) *loss = *n->hLoss;
  return LD_OK;
}

// Standalone tensor-core GEMM (bf16 bit patterns in, fp32 out) for tests:
// C[M x N] = A[M x K] * B[N x K]^T, M % 128 == 0, N % 64 == 0, K % 64 == 0.
extern "C" ld_status ld_tc_gemm(const uint16_t* A, const uint16_t* B, int32_t M, int32_t N, int32_t K, float* C,
                                int32_t device) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
  if (!A || !B || !C || M < 128 || M % 128 || N < 64 || N % 64 || K < 64 || K % 64)
    return ld_fail(LD_ERR_ARG, "shape must be M%%128, N%%64, K%%64");
  MLP_CUDA(cudaSetDevice(device));
  MLP_CUDA(gemm_init());
  void* mem = nullptr;
  const size_t ba = (size_t)M * K * 2, bb = (size_t)N * K * 2, bc = (size_t)M * N * 4;
  MLP_CUDA(cudaMalloc(&mem, ba + bb + bc + 256));
  char* p = (char*)mem;
  int* err = (int*)(p + ba + bb + bc);
  cudaError_t e = cudaMemcpy(p, A, ba, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(p + ba, B, bb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(err, 0, 4);
  if (e == cudaSuccess)
    e = gemm((const bf16*)p, (const bf16*)(p + ba), M, N, K, (float*)(p + ba + bb), nullptr, nullptr, nullptr, 0, err, 0);
  int h_err = 0;
  if (e == cudaSuccess) e = cudaMemcpy(C, p + ba + bb, bc, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&h_err, err, 4, cudaMemcpyDeviceToHost);
  cudaFree(mem);
  if (e != cudaSuccess) return ld_fail(LD_ERR_CUDA, "tensor-core GEMM: %s", cudaGetErrorString(e));
  if (h_err) return ld_fail(LD_ERR_TIMEOUT, "tensor-core GEMM wait ran out (code %d)", h_err);
  return LD_OK;
}
