// bf16 tensor-core GEMM on sm_100a (tcgen05 + TMEM) and the element-wise
// kernels of the proposal network's forward and backward passes.
//
//   C[M x N] = A[M x K] * B[N x K]^T      (A, B bf16, K-major; fp32 accumulate)
//
// One CTA (4 warps) computes a 128 x BN tile.  Per 64-wide K chunk the CTA
// copies the A and B tiles (cp.async, two stages) into shared memory in the
// canonical K-major layout without swizzle (8-row x 16-byte core matrices;
// core matrices 128 B apart along K, 1024 B apart along M/N), one elected
// thread issues four tcgen05.mma (K = 16 each) into a TMEM accumulator of
// 128 lanes x BN fp32 columns and commits them to the stage's mbarrier,
// which the CTA waits on before refilling that stage.  The epilogue reads the accumulator with
// tcgen05.ld (warp w owns lanes 32w..32w+31, i.e. rows 32w..32w+31 of the
// tile), optionally adds a bias and applies ReLU, and stores fp32 and/or
// bf16 (row-major and transposed) outputs.
//
// Every wait is bounded: a wait that runs out sets *err and the CTA stops
// issuing work; the host checks *err after the launch.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace ld {
namespace mlp {

constexpr int kTileM = 128;
constexpr int kTileK = 64;
constexpr unsigned kWaitLimit = 1u << 22;   // bounded mbarrier polls

enum : int { kErrWaitA = 1, kErrWaitB = 2 };

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// tcgen05 shared-memory matrix descriptor: K-major, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;                 // descriptor version for sm_100
  return d;                               // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor for kind::f16: bf16 x bf16 -> f32, both K-major
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
  return (1u << 4)                        // D format f32
       | (1u << 7)                        // A format bf16
       | (1u << 10)                       // B format bf16
       | ((uint32_t)(N >> 3) << 17)
       | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
  for (unsigned it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done) : "r"(mbar), "r"(phase) : "memory");
    if (done) return true;
  }
  return false;
}

struct GemmArgs {
  const __nv_bfloat16* A;   // M x K
  const __nv_bfloat16* B;   // N x K
  int M, N, K;
  float* C;                 // M x N fp32, or null
  __nv_bfloat16* H;         // M x N bf16 (bias + optional ReLU), or null
  __nv_bfloat16* HT;        // N x M bf16 transposed copy, or null
  const float* bias;        // N, or null
  int relu;
  int* err;
};

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory"); }

// Two-stage pipeline: while the tensor core multiplies chunk kc out of one
// shared-memory stage, the CTA's threads copy chunk kc + 1 into the other
// with cp.async.  A stage is refilled only after the mbarrier of the MMAs
// that read it has completed.
template <int BN>
__global__ void __launch_bounds__(128) tc_gemm_kernel(const GemmArgs g) {
  static_assert(BN == 64 || BN == 128 || BN == 256, "tile width");
  constexpr int kStageA = kTileM * kTileK * 2, kStageB = BN * kTileK * 2;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * BN;
  const uint32_t sbase = smem_u32(smem_raw);
  auto sA = [&](int st) { return sbase + st * (kStageA + kStageB); };
  auto sB = [&](int st) { return sbase + st * (kStageA + kStageB) + kStageA; };

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&tmem_base)), "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&mbar[0])), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&mbar[1])), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = instr_desc(kTileM, BN);

  // chunk kc of A (128 rows) and B (BN rows) into stage st, core-matrix layout:
  // row r, 16-byte piece c at ((r / 8) * 8 + c) * 128 + (r % 8) * 16
  auto load = [&](int kc, int st) {
    const int k0 = kc * kTileK;
#pragma unroll
    for (int i = 0; i < (kTileM * 8) / 128; ++i) {
      const int q = tid + 128 * i, r = q >> 3, c = q & 7;
      cp_async16(sA(st) + (((r >> 3) * 8 + c) * 128) + (r & 7) * 16, g.A + (size_t)(m0 + r) * g.K + k0 + c * 8);
    }
#pragma unroll
    for (int i = 0; i < (BN * 8) / 128; ++i) {
      const int q = tid + 128 * i, r = q >> 3, c = q & 7;
      cp_async16(sB(st) + (((r >> 3) * 8 + c) * 128) + (r & 7) * 16, g.B + (size_t)(n0 + r) * g.K + k0 + c * 8);
    }
    cp_async_commit();
  };

  const int nk = g.K / kTileK;
  bool ok = true;
  load(0, 0);
  for (int kc = 0; kc < nk; ++kc) {
    const int st = kc & 1;
    bool good = true;
    if (kc + 1 < nk) {
      // stage st ^ 1 was read by the MMAs of chunk kc - 1 (its ((kc-1)/2)-th use)
      if (kc >= 1) good = mbar_wait(smem_u32(&mbar[st ^ 1]), (uint32_t)((kc - 1) >> 1) & 1u);
      if (good) load(kc + 1, st ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    // generic-proxy shared-memory writes -> visible to the tensor core
    asm volatile("fence.proxy.async.shared::cta;");
    if (__syncthreads_or(!good)) { ok = false; break; }
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
      for (int kk = 0; kk < kTileK / 16; ++kk) {
        const uint64_t da = smem_desc(sA(st) + kk * 256, 128, 1024);
        const uint64_t db = smem_desc(sB(st) + kk * 256, 128, 1024);
        const uint32_t acc = (kc > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            :: "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   :: "r"(smem_u32(&mbar[st])));
    }
  }
  if (ok) {
    // the last commit tracks every MMA issued before it
    const bool done = mbar_wait(smem_u32(&mbar[(nk - 1) & 1]), (uint32_t)((nk - 1) >> 1) & 1u);
    ok = !__syncthreads_or(!done);
  } else {
    cp_async_wait<0>();
  }
  asm volatile("tcgen05.fence::after_thread_sync;");

  if (ok) {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
          "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
            "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
            "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;");
      float v[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        v[j] = __uint_as_float(r[j]);
        if (g.bias) v[j] += g.bias[n0 + c0 + j];
        if (g.relu) v[j] = fmaxf(v[j], 0.f);
      }
      if (g.C) {
        float4* dst = reinterpret_cast<float4*>(g.C + (size_t)row * g.N + n0 + c0);
#pragma unroll
        for (int j = 0; j < 4; ++j) dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
      }
      if (g.H) {
#pragma unroll
        for (int j = 0; j < 16; j += 2)
          *reinterpret_cast<__nv_bfloat162*>(g.H + (size_t)row * g.N + n0 + c0 + j) =
              __floats2bfloat162_rn(v[j], v[j + 1]);
      }
      if (g.HT) {
#pragma unroll
        for (int j = 0; j < 16; ++j) g.HT[(size_t)(n0 + c0 + j) * g.M + row] = __float2bfloat16_rn(v[j]);
      }
    }
  } else if (tid == 0) {
    atomicExch(g.err, kErrWaitA);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(BN));
  }
}

// ---- element-wise parts ---------------------------------------------------

// Step parameters read from device memory, so that one captured CUDA graph
// serves every training step: learning rate, Adam bias corrections
// 1 - beta1^t and 1 - beta2^t, and 1 / (number of unmasked targets).
enum { kHpLr = 0, kHpC1 = 1, kHpC2 = 2, kHpInvCount = 3, kHpWords = 4 };

// BCE with logits over valid entries: dz = (sigmoid(z) - t) * mask / count,
// written as bf16 (row-major and transposed); loss accumulated.  The logit
// is the network output plus `skip` times the input of the same index
// (a residual path without parameters; skip_x may be null).
__global__ void bce_grad_kernel(const float* z, const float* t, const float* mask, int rows, int cols,
                                const float* hp, const float* skip_x, float skip, __nv_bfloat16* dz,
                                __nv_bfloat16* dzT, float* loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const float inv_count = hp[kHpInvCount];
  float l = 0.f;
  if (i < rows * cols) {
    const int r = i / cols, c = i % cols;
    const float x = z[i] + (skip_x ? skip * skip_x[i] : 0.f), m = mask[i], y = t[i];
    const float s = 1.f / (1.f + expf(-x));
    const float g = (s - y) * m * inv_count;
    dz[i] = __float2bfloat16_rn(g);
    dzT[(size_t)c * rows + r] = __float2bfloat16_rn(g);
    // numerically stable log(1 + e^-|x|) + max(x, 0) - x y
    l = m * (fmaxf(x, 0.f) - x * y + log1pf(expf(-fabsf(x)))) * inv_count;
  }
  for (int off = 16; off > 0; off >>= 1) l += __shfl_xor_sync(0xffffffffu, l, off);
  if ((threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, l);
}

// dz = dh * (h > 0), bf16 row-major and / or transposed
__global__ void relu_grad_kernel(const float* dh, const __nv_bfloat16* h, int rows, int cols,
                                 __nv_bfloat16* dz, __nv_bfloat16* dzT) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const int r = i / cols, c = i % cols;
  const float g = __bfloat162float(h[i]) > 0.f ? dh[i] : 0.f;
  if (dz) dz[i] = __float2bfloat16_rn(g);
  if (dzT) dzT[(size_t)c * rows + r] = __float2bfloat16_rn(g);
}

// db[c] = sum over r of dzT[c][r] (bf16), one warp per output
__global__ void bias_grad_kernel(const __nv_bfloat16* dzT, int cols, int rows, float* db) {
  const int c = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= cols) return;
  float s = 0.f;
  for (int r = lane; r < rows; r += 32) s += __bfloat162float(dzT[(size_t)c * rows + r]);
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) db[c] = s;
}

// Adam on fp32 master weights w (rows x cols, gradient g); refreshes the
// bf16 copy wb and its transpose wbT (either may be null).  Learning rate
// and bias corrections come from the step parameters hp.
__global__ void adam_kernel(float* w, const float* g, float* m, float* v, int rows, int cols, const float* hp,
                            float b1, float b2, float eps, __nv_bfloat16* wb, __nv_bfloat16* wbT) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const float lr = hp[kHpLr], c1 = hp[kHpC1], c2 = hp[kHpC2];
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  const int r = i / cols, c = i % cols;
  if (wb) wb[i] = __float2bfloat16_rn(wi);
  if (wbT) wbT[(size_t)c * rows + r] = __float2bfloat16_rn(wi);
}

// fp32 -> bf16, optionally transposed (rows x cols -> cols x rows)
__global__ void to_bf16_kernel(const float* x, int rows, int cols, __nv_bfloat16* y, __nv_bfloat16* yT) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const int r = i / cols, c = i % cols;
  if (y) y[i] = __float2bfloat16_rn(x[i]);
  if (yT) yT[(size_t)c * rows + r] = __float2bfloat16_rn(x[i]);
}

}  // namespace mlp
}  // namespace ld
