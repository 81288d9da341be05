// Column-parallel enumeration kernel: any order d <= 10, up to 4096
// columns, int32 or int64 column sums.  It covers what the table kernel does
// not (d >= 4, wide matrices, entries whose sums need more than 32 bits).
//
// One warp walks one contiguous range of Gray indices (the worker split of
// calc_jmin_jmax, L_CUDA.cu:5-12, at warp granularity).  Lane l owns columns
// l, l+32, ...; each step moves one row between two messages (flips one
// sign for d == 1), as the reference kernels do (L_CUDA.cu:72-84, 111-123,
// 160-182, 218-238), but the column work is spread over the warp and the
// per-message |.|-sums are kept so only the two changed messages are summed
// again.  The step's row comes from an in-register base-d counter instead of
// the reference's 64-bit divisions.  A warp-shuffle reduction gives every
// labeling's value; the first index attaining the range's maximum is kept.
#pragma once
#include "common.cuh"

#ifndef LD_WIDE_MAXD
#define LD_WIDE_MAXD 10   // RANK_OF_NORM (functions.h:3)
#endif

namespace ld {

template <typename IT>
struct WideArgs {
  const IT* A;              // R x C row-major, row R-1 fixed (label 0 / +1)
  int R, C, d, marginal;
  unsigned long long n_begin, n_end;   // Gray indices of this launch
  // d >= 3 with label symmetry (sym_digits > 0): warps take the walks of
  // walk_len consecutive indices that pass the class-minimum test, by rank
  int sym_digits;                      // digits of the walk number
  unsigned long long walk_len;         // d^(R-1-sym_digits)
  const unsigned long long* sym_table; // completion counts (table_kernel.cuh walk_of_rank)
  unsigned long long rank_begin, rank_end;
  Reduce red;
};

constexpr int kWideThreads = 128;

template <typename IT>
__device__ __forceinline__ IT iabs(IT x) { return x < 0 ? -x : x; }

template <typename IT>
__device__ __forceinline__ long long warp_sum(IT v) {
  long long s = (long long)v;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  return s;
}

template <>
__device__ __forceinline__ long long warp_sum<int>(int v) {
  return (long long)__reduce_add_sync(0xffffffffu, v);
}

// labels of rows 0..R-2 for Gray index N (direct form)
__device__ __forceinline__ void direct_labels(unsigned long long N, int R, int d, int* lab) {
  if (d <= 2) {
    const unsigned long long g = N ^ (N >> 1);
    for (int i = 0; i < R - 1; ++i) lab[i] = (int)((g >> i) & 1ull);
  } else {
    unsigned long long q = N;
    const unsigned long long dd = (unsigned long long)d;
    for (int i = 0; i < R - 1; ++i) {
      const unsigned long long r = q % (2ull * dd);
      lab[i] = (int)(r < dd ? r : 2ull * dd - 1ull - r);
      q /= dd;
    }
  }
}

// MULTI = false: d == 1 (one signed vector, LM when marginal);
// MULTI = true:  d >= 2 (d message vectors).
// The labelings [lo, hi) walked by one warp in Gray order: seeded from
// lo's labels, then one row moved per index; (bv, bn) keeps the largest
// value and, among equal values, the first index.
template <typename IT, int PC, bool MULTI>
__device__ __forceinline__ void wide_range(const WideArgs<IT>& args, int lane, unsigned long long lo,
                                           unsigned long long hi, long long& bv, unsigned long long& bn) {
  const int R = args.R, C = args.C, d = args.d;
  if (lo < hi) {
    int lab[64];
    int dig[65];
    direct_labels(lo, R, d, lab);
    const IT* A = args.A;
    IT s[MULTI ? LD_WIDE_MAXD : 1][PC];
    long long part[MULTI ? LD_WIDE_MAXD : 1];
#pragma unroll
    for (int t = 0; t < PC; ++t) {
      const int l = lane + 32 * t;
      const IT fixed = l < C ? A[(size_t)(R - 1) * C + l] : (IT)0;
      s[0][t] = fixed;
      if (MULTI) for (int m = 1; m < d; ++m) s[m][t] = 0;
    }
    for (int i = 0; i < R - 1; ++i) {
#pragma unroll
      for (int t = 0; t < PC; ++t) {
        const int l = lane + 32 * t;
        const IT x = l < C ? A[(size_t)i * C + l] : (IT)0;
        if (MULTI) s[lab[i]][t] += x;
        else s[0][t] += lab[i] ? x : -x;
      }
    }
    long long val_lane = 0;
    if (MULTI) {
      for (int m = 0; m < d; ++m) {
        IT acc = 0;
#pragma unroll
        for (int t = 0; t < PC; ++t) acc += iabs(s[m][t]);
        part[m] = (long long)acc;
        val_lane += part[m];
      }
    } else {
      IT acc = 0;
#pragma unroll
      for (int t = 0; t < PC; ++t)
        acc += (args.marginal && lane == 0 && t == 0) ? s[0][t] : iabs(s[0][t]);
      val_lane = (long long)acc;
    }
    long long v = warp_sum<long long>(val_lane);
    if (v > bv) { bv = v; bn = lo; }
    // base-d digits of lo for the step search (d >= 3)
    const int dd = d <= 2 ? 2 : d;
    int dsum = 0;
    {
      unsigned long long q = lo;
      for (int i = 0; i < 65; ++i) { dig[i] = (int)(q % (unsigned long long)dd); dsum ^= dig[i] & 1; q /= (unsigned long long)dd; }
    }
    for (unsigned long long N = lo + 1; N < hi; ++N) {
      int i, a, b;
      if (d <= 2) {
        i = __ffsll((long long)N) - 1;
        b = (int)(((N >> (i + 1)) & 1ull) ^ 1ull);
        a = b ^ 1;
      } else {
        i = 0;
        while (dig[i] == dd - 1) { dig[i] = 0; ++i; }
        dig[i] += 1;
        dsum ^= 1;
        const int par = (dd & 1) ? ((dsum ^ dig[i]) & 1) : (dig[i + 1] & 1);
        b = par ? dd - 1 - dig[i] : dig[i];
        a = lab[i];
      }
      lab[i] = b;
      const IT* row = A + (size_t)i * C;
      if (MULTI) {
        IT pa = 0, pb = 0;
#pragma unroll
        for (int t = 0; t < PC; ++t) {
          const int l = lane + 32 * t;
          const IT x = l < C ? row[l] : (IT)0;
          s[a][t] -= x;
          s[b][t] += x;
          pa += iabs(s[a][t]);
          pb += iabs(s[b][t]);
        }
        val_lane += (long long)pa - part[a] + (long long)pb - part[b];
        part[a] = pa; part[b] = pb;
      } else {
        IT acc = 0;
#pragma unroll
        for (int t = 0; t < PC; ++t) {
          const int l = lane + 32 * t;
          const IT x = l < C ? row[l] : (IT)0;
          s[0][t] += b ? (IT)(2 * x) : (IT)(-2 * x);
          acc += (args.marginal && lane == 0 && t == 0) ? s[0][t] : iabs(s[0][t]);
        }
        val_lane = (long long)acc;
      }
      v = warp_sum<long long>(val_lane);
      if (v > bv) { bv = v; bn = N; }
    }
  }
}

// The passing walk of rank i for a runtime order D (the device copy of
// walk_of_rank in table_kernel.cuh, and of symmetry.c's host copy).
static __device__ __forceinline__ unsigned long long walk_of_rank_rt(unsigned long long i, int P, int D,
                                                                  const unsigned long long* __restrict__ f) {
  unsigned used = 1u;
  int seen = 1, par = 0, q = P - 1;
  unsigned long long w = 0;
  for (; q >= 0 && seen < D - 1; --q) {
    const unsigned unused = ~used & ((1u << D) - 1u);
    const int want = par ? 31 - __clz((int)unused) : __ffs((int)unused) - 1;
    int n = 0, lab = 0, np = 0;
    for (; n < D; ++n) {
      lab = par ? D - 1 - n : n;
      if (!(((used >> lab) & 1u) || lab == want)) continue;
      np = (D & 1) ? (par ^ (n & 1)) : (n & 1);
      const unsigned long long c = __ldg(f + ((size_t)((used | (1u << lab)) >> 1) * 2 + np) * (size_t)(P + 1) + q);
      if (i < c) break;
      i -= c;
    }
    if (n == D) { n = D - 1; lab = par ? 0 : D - 1; np = (D & 1) ? (par ^ (n & 1)) : (n & 1); }  // i past the end
    w = w * (unsigned long long)D + (unsigned long long)n;
    if (!((used >> lab) & 1u)) { used |= 1u << lab; ++seen; }
    par = np;
  }
  for (int t = 0; t <= q; ++t) w *= (unsigned long long)D;
  return w + i;
}

template <typename IT, int PC, bool MULTI, bool SYM = false>
__global__ void __launch_bounds__(kWideThreads) wide_kernel(const WideArgs<IT> args) {
  const int lane = threadIdx.x & 31;
  const unsigned long long gw = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nw = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  long long bv = LLONG_MIN;
  unsigned long long bn = ULLONG_MAX;
  if constexpr (SYM) {
    // label symmetry: the passing walks by rank, in increasing index order
    // per warp
    for (unsigned long long r = args.rank_begin + gw; r < args.rank_end; r += nw) {
      const unsigned long long lo = walk_of_rank_rt(r, args.sym_digits, args.d, args.sym_table) * args.walk_len;
      wide_range<IT, PC, MULTI>(args, lane, lo, lo + args.walk_len, bv, bn);
    }
  } else {
    // one contiguous range per warp
    const unsigned long long n = args.n_end - args.n_begin;
    const unsigned long long steps = n / nw, rem = n % nw;
    const unsigned long long lo = args.n_begin + gw * steps + (gw < rem ? gw : rem);
    const unsigned long long hi = lo + steps + (gw < rem ? 1ull : 0ull);
    wide_range<IT, PC, MULTI>(args, lane, lo, hi, bv, bn);
  }
  // one candidate per warp: lane 0's copy (all lanes agree)
  if (lane != 0) { bv = LLONG_MIN; bn = ULLONG_MAX; }
  grid_reduce(bv, bn, args.red);
}

}  // namespace ld
