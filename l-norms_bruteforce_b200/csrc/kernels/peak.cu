// INT32 issue roofline microbenchmark.
//
// Every thread runs 8 independent dependency chains x <- (x + y) ^ z.  An add
// and an xor cannot be fused into one instruction, and the recurrence has no
// closed form, so each counted operation is one executed 32-bit integer ALU
// instruction per lane.  The measured rate is the denominator of the
// enumeration kernels' integer roofline.
#include <cuda_runtime.h>

#include "../host/ld_internal.h"
#include "../abi/device_guard.h"

namespace {

__global__ void __launch_bounds__(256) int32_peak_kernel(int* sink, int iters, int seed) {
  int x0 = (int)threadIdx.x + seed, x1 = x0 * 3, x2 = x0 * 5, x3 = x0 * 7;
  int x4 = x0 * 11, x5 = x0 * 13, x6 = x0 * 17, x7 = x0 * 19;
  const int y = seed * 31 + 7, z = seed * 17 + 3;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      x0 = (x0 + y) ^ z; x1 = (x1 + y) ^ z; x2 = (x2 + y) ^ z; x3 = (x3 + y) ^ z;
      x4 = (x4 + y) ^ z; x5 = (x5 + y) ^ z; x6 = (x6 + y) ^ z; x7 = (x7 + y) ^ z;
    }
  }
  const int r = x0 ^ x1 ^ x2 ^ x3 ^ x4 ^ x5 ^ x6 ^ x7;
  if (r == 0x7fffffff) sink[blockIdx.x] = r;   // keeps the chains live
}

}  // namespace

// ops per launch = blocks * 256 threads * iters * 8 unroll * 8 chains * 2 ops
extern "C" ld_status ld_measure_int32_peak(int32_t device, double* ops_per_second, double* ms) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
  if (!ops_per_second) return ld_fail(LD_ERR_ARG, "null output");
  if (cudaSetDevice(device) != cudaSuccess) return ld_fail(LD_ERR_NODEV, "no device %d", device);
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return ld_fail(LD_ERR_NODEV, "no device %d", device);
  const int blocks = p.multiProcessorCount * 8, threads = 256, iters = 4096;
  int* sink = nullptr;
  cudaEvent_t e0, e1;
  if (cudaMalloc(&sink, sizeof(int) * blocks) != cudaSuccess) return ld_fail(LD_ERR_CUDA, "cudaMalloc failed");
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 6; ++rep) {
    cudaEventRecord(e0);
    int32_peak_kernel<<<blocks, threads>>>(sink, iters, rep + 1);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    if (rep > 0 && t < best) best = t;   // first launch is warm-up
  }
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (err != cudaSuccess) return ld_fail(LD_ERR_CUDA, "peak kernel: %s", cudaGetErrorString(err));
  const double ops = (double)blocks * threads * iters * 8.0 * 8.0 * 2.0;
  *ops_per_second = ops / (best * 1e-3);
  if (ms) *ms = best;
  return LD_OK;
}
