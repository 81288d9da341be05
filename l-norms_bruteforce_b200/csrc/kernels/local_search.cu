// Single-row-move local search: polish starting labelings into an
// incumbent for the pruned search.
//
// One warp per start.  The warp keeps the message column sums S_m (int64)
// and the labels in shared memory; each round every lane evaluates the gain
// of every move of its rows (d = 1: flip the sign; d >= 2: move the row to
// another message), the warp takes the largest gain (ties: smallest row,
// then smallest label) and applies it, until no move gains or the round
// limit is reached.  The last row keeps its fixed label (+1 / message 0), as
// in the enumeration.  Values are exact int64; a start's final value is the
// value of its final labeling.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "../abi/smem_limit.h"
#include "../host/ld_internal.h"
#include "../abi/device_guard.h"

namespace {

constexpr int kLsWarps = 4;
constexpr int kLsMaxCols = 128;
constexpr int kLsMaxRows = 64;

struct LsArgs {
  const long long* A;     // R x C
  int R, C, d, marginal;
  const int* starts;      // n x (R-1) labels
  int n, max_rounds;
  long long* values;      // n
  int* labels;            // n x (R-1)
};

__device__ __forceinline__ long long labs64(long long x) { return x < 0 ? -x : x; }

// The block's warps share one copy of the matrix in shared memory (dynamic,
// R x C int64), staged once: every round of every start reads it.
__global__ void __launch_bounds__(kLsWarps * 32) local_search_kernel(const LsArgs a) {
  extern __shared__ long long sA[];
  __shared__ long long sS[kLsWarps][3][kLsMaxCols];
  __shared__ int sLab[kLsWarps][kLsMaxRows];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int t = threadIdx.x; t < a.R * a.C; t += blockDim.x) sA[t] = a.A[t];
  __syncthreads();
  const int start = blockIdx.x * kLsWarps + wid;
  if (start >= a.n) return;
  const int R = a.R, C = a.C, d = a.d, nm = d == 1 ? 1 : d;
  long long (*S)[kLsMaxCols] = sS[wid];
  int* lab = sLab[wid];
  for (int i = lane; i < R - 1; i += 32) lab[i] = a.starts[(size_t)start * (R - 1) + i];
  if (lane == 0) lab[R - 1] = d == 1 ? 1 : 0;
  __syncwarp();
  for (int l = lane; l < C; l += 32) {
    for (int m = 0; m < nm; ++m) S[m][l] = 0;
    for (int i = 0; i < R; ++i) {
      const long long x = sA[i * C + l];
      if (d == 1) S[0][l] += lab[i] ? x : -x;
      else S[lab[i]][l] += x;
    }
  }
  __syncwarp();
  for (int round = 0; round < a.max_rounds; ++round) {
    long long bg = 0;           // best gain of this lane (> 0 to count)
    int bi = INT_MAX, bt = 0;
    for (int i = lane; i < R - 1; i += 32) {
      const long long* row = sA + i * C;
      if (d == 1) {
        const long long sg = lab[i] ? -2 : 2;   // change of the column sum per unit of A
        long long g = 0;
        for (int l = 0; l < C; ++l) {
          const long long s = S[0][l], ns = s + sg * row[l];
          g += (a.marginal && l == 0) ? ns - s : labs64(ns) - labs64(s);
        }
        if (g > bg || (g == bg && g > 0 && i < bi)) { bg = g; bi = i; bt = lab[i] ^ 1; }
      } else {
        const int from = lab[i];
        for (int t = 0; t < d; ++t) {
          if (t == from) continue;
          long long g = 0;
          for (int l = 0; l < C; ++l) {
            const long long x = row[l], sf = S[from][l], st = S[t][l];
            g += labs64(sf - x) + labs64(st + x) - labs64(sf) - labs64(st);
          }
          if (g > bg || (g == bg && g > 0 && (i < bi || (i == bi && t < bt)))) { bg = g; bi = i; bt = t; }
        }
      }
    }
    // warp argmax: largest gain, then smallest row, then smallest label
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const long long og = __shfl_xor_sync(0xffffffffu, bg, off);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
      const int ot = __shfl_xor_sync(0xffffffffu, bt, off);
      if (og > bg || (og == bg && (oi < bi || (oi == bi && ot < bt)))) { bg = og; bi = oi; bt = ot; }
    }
    if (bg <= 0 || bi == INT_MAX) break;
    const int from = lab[bi];
    __syncwarp();
    for (int l = lane; l < C; l += 32) {
      const long long x = sA[bi * C + l];
      if (d == 1) S[0][l] += bt ? 2 * x : -2 * x;
      else { S[from][l] -= x; S[bt][l] += x; }
    }
    if (lane == 0) lab[bi] = bt;
    __syncwarp();
  }
  long long v = 0;
  for (int l = lane; l < C; l += 32)
    for (int m = 0; m < nm; ++m) v += (d == 1 && a.marginal && l == 0) ? S[m][l] : labs64(S[m][l]);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if (lane == 0) a.values[start] = v;
  for (int i = lane; i < R - 1; i += 32) a.labels[(size_t)start * (R - 1) + i] = lab[i];
}

#define LS_CUDA(call)                                                                \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) return ld_fail(LD_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

// Per-device workspace kept between calls: one device arena, one pinned
// staging buffer (inputs out, results back in one copy each) and a stream.
struct LsWorkspace {
  char* dmem = nullptr;
  size_t dcap = 0;
  char* hmem = nullptr;
  size_t hcap = 0;
  cudaStream_t stream = nullptr;
};
std::mutex g_ls_mu[64];
LsWorkspace g_ls[64];

size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" ld_status ld_local_search(const int64_t* a, int32_t R, int32_t C, int32_t d, int32_t marginal,
                                     const int32_t* starts, int32_t n, int32_t max_rounds, int32_t device,
                                     int64_t* values, int32_t* labels) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
  if (!a || !starts || !values || !labels || n < 1 || R < 2 || C < 1)
    return ld_fail(LD_ERR_ARG, "bad local-search arguments");
  if (d < 1 || d > 3 || C > kLsMaxCols || R > kLsMaxRows)
    return ld_fail(LD_ERR_LIMIT, "local search takes d <= 3, <= %d columns, <= %d rows", kLsMaxCols, kLsMaxRows);
  if (device < 0 || device >= 64) return ld_fail(LD_ERR_ARG, "device %d out of range", device);
  for (int64_t t = 0; t < (int64_t)n * (R - 1); ++t)
    if (starts[t] < 0 || starts[t] >= (d == 1 ? 2 : d)) return ld_fail(LD_ERR_ARG, "start label out of range");
  const size_t nl = (size_t)n * (R - 1);
  // inputs: matrix | starts; results: values | labels
  const size_t bA = up256(sizeof(long long) * (size_t)R * C), bS = up256(sizeof(int) * nl);
  const size_t bV = up256(sizeof(long long) * (size_t)n), bL = up256(sizeof(int) * nl);
  const size_t in_bytes = bA + bS, out_bytes = bV + bL, total = in_bytes + out_bytes;
  if (cudaSetDevice(device) != cudaSuccess) return ld_fail(LD_ERR_NODEV, "no device %d", device);
  std::lock_guard<std::mutex> lock(g_ls_mu[device]);
  LsWorkspace& w = g_ls[device];
  if (!w.stream) LS_CUDA(cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking));
  if (w.dcap < total) {
    if (w.dmem) { LS_CUDA(cudaStreamSynchronize(w.stream)); LS_CUDA(cudaFree(w.dmem)); w.dmem = nullptr; w.dcap = 0; }
    LS_CUDA(cudaMalloc(&w.dmem, total));
    w.dcap = total;
  }
  if (w.hcap < total) {
    if (w.hmem) { LS_CUDA(cudaStreamSynchronize(w.stream)); LS_CUDA(cudaFreeHost(w.hmem)); w.hmem = nullptr; w.hcap = 0; }
    LS_CUDA(cudaMallocHost(&w.hmem, total));
    w.hcap = total;
  }
  memcpy(w.hmem, a, sizeof(long long) * (size_t)R * C);
  memcpy(w.hmem + bA, starts, sizeof(int) * nl);
  LS_CUDA(cudaMemcpyAsync(w.dmem, w.hmem, in_bytes, cudaMemcpyHostToDevice, w.stream));
  LsArgs args{(const long long*)w.dmem, R, C, d, marginal, (const int*)(w.dmem + bA), n,
              max_rounds > 0 ? max_rounds : 4 * R, (long long*)(w.dmem + in_bytes),
              (int*)(w.dmem + in_bytes + bV)};
  const size_t smem = sizeof(long long) * (size_t)R * C;   // at most 64 rows x 128 columns = 64 KB
  if (ld_raise_smem_limit((const void*)local_search_kernel, smem) != cudaSuccess)
    return ld_fail(LD_ERR_CUDA, "local search: cannot reserve %zu bytes of shared memory", smem);
  local_search_kernel<<<(n + kLsWarps - 1) / kLsWarps, kLsWarps * 32, smem, w.stream>>>(args);
  LS_CUDA(cudaGetLastError());
  LS_CUDA(cudaMemcpyAsync(w.hmem + in_bytes, w.dmem + in_bytes, out_bytes, cudaMemcpyDeviceToHost, w.stream));
  LS_CUDA(cudaStreamSynchronize(w.stream));
  memcpy(values, w.hmem + in_bytes, sizeof(long long) * (size_t)n);
  memcpy(labels, w.hmem + in_bytes + bV, sizeof(int) * nl);
  return LD_OK;
}
