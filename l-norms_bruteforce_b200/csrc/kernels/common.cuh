// Device-side pieces shared by the enumeration kernels: packed integer lanes,
// the (value, Gray index) order, and the grid-wide reduction that turns
// per-thread maxima into the norm and the smallest Gray index attaining it
// (the reference's strict '>' inside a worker, L_CUDA.cu:80, and strict '<'
// across workers in index order, L_CUDA.cu:347).
#pragma once
#include <cstdint>
#include <climits>

namespace ld {

// One block's (or the final) candidate.
struct Slot {
  long long value;          // norm candidate (LLONG_MIN = none)
  unsigned long long index; // its Gray index (ULLONG_MAX = none)
};

// Scratch a launch reduces through.  `slots` holds one entry per block;
// `counter` and `gvalue` must be 0 / LLONG_MIN before the first launch and
// are restored by the last block of every launch.
struct Reduce {
  Slot* slots;
  unsigned int* counter;
  long long* gvalue;
  Slot* result;
  unsigned long long* work;   // walk counter the launch's warps fetch from (0 before
                              // the launch, reset by the last block), or null
};

// ---- packed integer lanes ----------------------------------------------
// PK columns share one 32-bit word as independent signed lanes of 32/PK
// bits.  The host picks PK from an exact bound on every partial column sum,
// so lane arithmetic never wraps.  Only 32-bit and 8x4-bit lanes exist:
// vabsdiff4 runs at the rate of a 32-bit absolute difference on sm_100a and
// covers four columns, while the 16x2-bit form measured about seven times
// slower than two 32-bit ones.
template <int PK> struct Lanes;

template <> struct Lanes<1> {
  __device__ __forceinline__ static uint32_t add(uint32_t a, uint32_t b) { return a + b; }
  __device__ __forceinline__ static uint32_t sub(uint32_t a, uint32_t b) { return a - b; }
  // c + |a - b|, a and b signed 32-bit
  __device__ __forceinline__ static uint32_t sad(uint32_t a, uint32_t b, uint32_t c) {
    return __sad((int)a, (int)b, c);
  }
};

template <> struct Lanes<4> {
  __device__ __forceinline__ static uint32_t add(uint32_t a, uint32_t b) { return __vadd4(a, b); }
  __device__ __forceinline__ static uint32_t sub(uint32_t a, uint32_t b) { return __vsub4(a, b); }
  // c + sum over the 4 bytes of |a.b_i - b.b_i|, bytes signed 8-bit
  __device__ __forceinline__ static uint32_t sad(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t d;
    asm("vabsdiff4.u32.s32.s32.add %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
  }
};

// ---- candidate order ----------------------------------------------------
__device__ __forceinline__ bool better(long long v, unsigned long long n,
                                       long long bv, unsigned long long bn) {
  return v > bv || (v == bv && n < bn);
}

__device__ __forceinline__ void warp_best(long long& v, unsigned long long& n) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    long long ov = __shfl_xor_sync(0xffffffffu, v, off);
    unsigned long long on = __shfl_xor_sync(0xffffffffu, n, off);
    if (better(ov, on, v, n)) { v = ov; n = on; }
  }
}

// Block-wide best, then one atomicMax per block on the value and a slot
// write; the last block to finish picks the smallest index among the slots
// that reach the maximum and re-arms the scratch for the next launch.
// Must be called by every thread of the block.
__device__ __forceinline__ void grid_reduce(long long v, unsigned long long n, const Reduce& R) {
  __shared__ long long s_v[32];
  __shared__ unsigned long long s_n[32];
  __shared__ bool s_last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
  warp_best(v, n);
  if (lane == 0) { s_v[wid] = v; s_n[wid] = n; }
  __syncthreads();
  if (wid == 0) {
    v = lane < nwarps ? s_v[lane] : LLONG_MIN;
    n = lane < nwarps ? s_n[lane] : ULLONG_MAX;
    warp_best(v, n);
    if (lane == 0) {
      R.slots[blockIdx.x].value = v;
      R.slots[blockIdx.x].index = n;
      if (v != LLONG_MIN) atomicMax(R.gvalue, v);
      __threadfence();
      unsigned int done = atomicAdd(R.counter, 1u);
      s_last = (done == gridDim.x - 1);
    }
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  const long long gmax = *((volatile long long*)R.gvalue);
  unsigned long long bn = ULLONG_MAX;
  for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    long long sv = __ldcg(&R.slots[b].value);
    unsigned long long sn = __ldcg(&R.slots[b].index);
    if (sv == gmax && sn < bn) bn = sn;
  }
  long long vv = gmax;
  warp_best(vv, bn);
  __syncthreads();
  if (lane == 0) { s_v[wid] = vv; s_n[wid] = bn; }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long best = ULLONG_MAX;
    for (int w = 0; w < nwarps; ++w) if (s_n[w] < best) best = s_n[w];
    R.result->value = gmax;
    R.result->index = best;
    *R.gvalue = LLONG_MIN;
    *R.counter = 0u;
    if (R.work) *R.work = 0ull;   // every block has finished fetching walks
    __threadfence();
  }
}

}  // namespace ld
