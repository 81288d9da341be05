// Batched exact solves: a persistent kernel that takes (matrix, walk range)
// chunks from a device work queue.
//
// Every CTA loops: one atomicAdd on the queue head hands it the next chunk;
// when the chunk's matrix differs from the one the CTA has staged, the CTA
// stages that matrix's packed rows and builds its table in shared memory;
// then its threads walk the chunk's walks exactly as the table kernel does
// (table_kernel.cuh) and the CTA writes the chunk's best (value, smallest
// Gray index) to the chunk's slot.  A second kernel folds each matrix's
// chunk slots into its result.  Chunks of one matrix are consecutive in
// the queue, largest matrices first, so CTAs restage rarely and the queue
// drains evenly.
#pragma once
#include "table_kernel.cuh"

namespace ld {

struct BatchProblem {
  const uint32_t* A;        // R x WT packed rows
  const uint32_t* tot;      // WT words
  const uint32_t* hinit;    // WT words
  const uint32_t* tbias;    // WT words
  int R, k, B, fw;
  int sym_digits;           // D = 3: walk-number digits of the label-symmetry test (0 = off)
  unsigned long long walk_len;
  unsigned long long sym_pw;  // 3^(sym_digits - 1)
  long long value_offset;
};

struct BatchChunk {
  unsigned long long walk_begin, walk_end;
  int problem;
  int pad;
};

struct BatchArgs {
  const BatchProblem* problems;
  const BatchChunk* chunks;
  int nchunks;
  unsigned int* head;       // queue head, 0 before the launch
  Slot* chunk_results;      // one per chunk
};

// Threads per CTA: the autotuner picks 64 or 128 per lane class (the
// kernels read blockDim); 128 is the default and the launch bound.  A bound
// of 256 (to offer 256-thread CTAs) changed the register allocation of the
// int32 classes (48 words: 127 -> 164 registers, a resident CTA less per
// SM) and cost 2.5 % of the batch replay, more than the larger CTAs gained.
constexpr int kBatchThreads = 128;
constexpr int kBatchMaxThreads = 128;

// block-wide (max value, smallest index); the result is valid in thread 0
__device__ __forceinline__ void block_best(long long& v, unsigned long long& n) {
  __shared__ long long s_v[32];
  __shared__ unsigned long long s_n[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
  warp_best(v, n);
  __syncthreads();
  if (lane == 0) { s_v[wid] = v; s_n[wid] = n; }
  __syncthreads();
  if (wid == 0) {
    v = lane < nwarps ? s_v[lane] : LLONG_MIN;
    n = lane < nwarps ? s_n[lane] : ULLONG_MAX;
    warp_best(v, n);
  }
}

// Table entry j (the low rows' partial sums for low labeling j, in Gray
// order) of a D-vector problem, written to e.
template <int D, int WB, int WA>
__device__ __forceinline__ void batch_build_entry(int j, int k, const uint32_t* sA, const uint32_t* sTot,
                                                  const uint32_t* sTb, uint32_t* e) {
  using S = Shape<D, WB, WA>;
  constexpr int WT = S::WT, WV = S::WV;
  uint32_t L1[WV], L2[WV];
#pragma unroll
  for (int w = 0; w < WV; ++w) { L1[w] = D == 1 ? sTb[w] : 0u; L2[w] = 0u; }
  if (D <= 2) {
    const unsigned g = (unsigned)j ^ ((unsigned)j >> 1);
    for (int i = 0; i < k; ++i) {
      const int lab = (g >> i) & 1u;
      const uint32_t* row = sA + i * WT;
      if (D == 1) {
#pragma unroll
        for (int w = 0; w < WV; ++w) L1[w] = lab ? wsub<WB>(w, L1[w], row[w]) : wadd<WB>(w, L1[w], row[w]);
      } else if (lab) {
#pragma unroll
        for (int w = 0; w < WV; ++w) L1[w] = wadd<WB>(w, L1[w], row[w]);
      }
    }
  } else {
    unsigned q = (unsigned)j;
    for (int i = 0; i < k; ++i) {
      const unsigned r = q % 6u;
      const int lab = r < 3u ? (int)r : 5 - (int)r;
      q /= 3u;
      const uint32_t* row = sA + i * WT;
      if (lab == 1) {
#pragma unroll
        for (int w = 0; w < WV; ++w) L1[w] = wadd<WB>(w, L1[w], row[w]);
      } else if (lab == 2) {
#pragma unroll
        for (int w = 0; w < WV; ++w) L2[w] = wadd<WB>(w, L2[w], row[w]);
      }
    }
  }
#pragma unroll
  for (int w = 0; w < WT; ++w) {
    if (w < WV) {
      if (D == 1) {
        e[w] = L1[w];
      } else if (D == 2) {
        e[w] = wsub<WB>(w, 0u, L1[w]);
        e[WT + w] = wsub<WB>(w, sTot[w], L1[w]);
      } else {
        e[w] = wsub<WB>(w, 0u, L1[w]);
        e[WT + w] = wsub<WB>(w, 0u, L2[w]);
        e[2 * WT + w] = wsub<WB>(w, wsub<WB>(w, sTot[w], L1[w]), L2[w]);
      }
    } else {
#pragma unroll
      for (int v = 0; v < D; ++v) e[v * WT + w] = 0u;
    }
  }
}

template <int D, int WB, int WA>
__global__ void __launch_bounds__(kBatchMaxThreads) batch_table_kernel(const BatchArgs args) {
  using S = Shape<D, WB, WA>;
  constexpr int WT = S::WT, WV = S::WV, NW = S::NW;
  extern __shared__ __align__(16) uint32_t smem[];
  __shared__ int s_chunk;
  int loaded = -1;
  uint32_t H[S::NR * WV];
  for (;;) {
    if (threadIdx.x == 0) s_chunk = (int)atomicAdd(args.head, 1u);
    __syncthreads();
    const int c = s_chunk;
    __syncthreads();
    if (c >= args.nchunks) break;
    const BatchChunk ch = args.chunks[c];
    const BatchProblem pr = args.problems[ch.problem];
    const int R = pr.R, k = pr.k, B = pr.B, nh = R - 1 - k;
    uint32_t* sA = smem;
    uint32_t* sTot = sA + R * WT;
    uint32_t* sH0 = sTot + WT;
    uint32_t* sTb = sH0 + WT;
    uint32_t* sT = smem + (((R * WT + 3 * WT) + 3) & ~3);
    if (ch.problem != loaded) {
      for (int t = threadIdx.x; t < R * WT; t += blockDim.x) sA[t] = pr.A[t];
      for (int t = threadIdx.x; t < WT; t += blockDim.x) {
        sTot[t] = pr.tot[t];
        sH0[t] = pr.hinit[t];
        sTb[t] = pr.tbias[t];
      }
      __syncthreads();
      for (int j = threadIdx.x; j < B; j += blockDim.x)
        batch_build_entry<D, WB, WA>(j, k, sA, sTot, sTb, sT + j * NW);
      __syncthreads();
      loaded = ch.problem;
    }
    const unsigned long long WL = pr.walk_len;
    int best = INT_MIN;
    unsigned long long best_h = 0ull;
    for (unsigned long long wk = ch.walk_begin + threadIdx.x; wk < ch.walk_end; wk += blockDim.x) {
      if constexpr (D == 3) {   // walks holding no class minimum (table_kernel.cuh)
        if (pr.sym_digits > 0 && !walk_holds_class_min<3>(wk, pr.sym_digits, pr.sym_pw)) continue;
      }
      const unsigned long long h0 = wk * WL;
      seed_high<D, WB, WA>(H, sA, sH0, k, nh, h0);
      for (unsigned long long u = 0; u < WL; ++u) {
        if (u) {
          const unsigned long long h = h0 + u;
          int i, a, b;
          if (D <= 2) {
            i = __ffsll((long long)u) - 1;
            b = (int)(((h >> (i + 1)) & 1ull) ^ 1ull);
            a = b ^ 1;
          } else {
            unsigned long long q = u;
            i = 0;
            while (q % 3ull == 0ull) { q /= 3ull; ++i; }
            const int cc = (int)(q % 3ull);
            const int par = (int)((wk ^ (q / 3ull)) & 1ull);
            b = par ? 2 - cc : cc;
            a = par ? 3 - cc : cc - 1;
          }
          move_row<D, WB, WA>(H, sA + (k + i) * WT, a, b);
        }
        const int m = scan_max<D, WB, WA>(H, sT, B);
        if (m > best) { best = m; best_h = h0 + u; }
      }
    }
    long long bv = LLONG_MIN;
    unsigned long long bn = ULLONG_MAX;
    if (best != INT_MIN) {
      seed_high<D, WB, WA>(H, sA, sH0, k, nh, best_h);
      const bool rev = (best_h & 1ull) != 0ull;
      for (int jj = 0; jj < B; ++jj) {
        const int je = rev ? B - 1 - jj : jj;
        if (entry_value<D, WB, WA>(H, sT + je * NW) == best) {
          bn = best_h * (unsigned long long)B + (unsigned long long)jj;
          break;
        }
      }
      bv = (long long)best - pr.value_offset;
    }
    block_best(bv, bn);
    if (threadIdx.x == 0) { args.chunk_results[c].value = bv; args.chunk_results[c].index = bn; }
  }
}

// ---- column-split instances ------------------------------------------------
//
// Wide int32 classes (WB >= 40 words, no 8-bit words): two adjacent threads
// share one high index, each holding half of the columns.  Each half is a
// Shape<D, WB/2, 0> problem on its own copy of half the rows, totals and
// table in shared memory; an entry's value is the sum of the two halves'
// (one shuffle within the pair).  A thread then holds half the register
// vectors and loads half of each entry, which lets more warps stay resident
// on the register file.  The halves' shared-memory regions are staggered by
// 16 bytes when they would otherwise start on the same bank, so the pair's
// two table reads are served in one pass.

__host__ __device__ constexpr bool batch_split_class(int WB, int WA) { return WA == 0 && WB >= 40 && WB % 8 == 0; }

// words of one half's region: rows, totals, initial H, table bias, table
__host__ __device__ inline int batch_split_span(int D, int WB, int R, int B) {
  const int WH = WB / 2;
  const int head = ((R * WH + 3 * WH) + 3) & ~3;
  int span = head + B * D * WH;
  if ((span & 31) == 0) span += 4;
  return span;
}

__host__ __device__ inline int batch_split_smem_words(int D, int WB, int R, int B) {
  return 2 * batch_split_span(D, WB, R, B);
}

// max over the B entries of (this half's value + the partner half's)
template <int D, int WH>
__device__ __forceinline__ int scan_max_split(const uint32_t* H, const uint32_t* sT, int B, unsigned pair) {
  using S = Shape<D, WH, 0>;
  int m = INT_MIN;
  int j = 0;
  for (; j + 2 <= B; j += 2) {
    const uint4* t0 = reinterpret_cast<const uint4*>(sT + j * S::NW);
    const uint4* t1 = reinterpret_cast<const uint4*>(sT + (j + 1) * S::NW);
    uint32_t a0 = 0u, a1 = 0u, b0 = 0u, b1 = 0u;
#pragma unroll
    for (int q = 0; q < S::NW / 4; ++q) {
      sad4<D, WH, 0>(H, t0[q], q, a0, a1);
      sad4<D, WH, 0>(H, t1[q], q, b0, b1);
    }
    int v0 = (int)(a0 + a1), v1 = (int)(b0 + b1);
    v0 += __shfl_xor_sync(pair, v0, 1);
    v1 += __shfl_xor_sync(pair, v1, 1);
    m = max(m, max(v0, v1));
  }
  if (j < B) {
    int v = entry_value<D, WH, 0>(H, sT + j * S::NW);
    v += __shfl_xor_sync(pair, v, 1);
    m = max(m, v);
  }
  return m;
}

template <int D, int WB>
__global__ void __launch_bounds__(kBatchMaxThreads) batch_split_kernel(const BatchArgs args) {
  static_assert(batch_split_class(WB, 0), "split classes: int32 words only, WB >= 40, a multiple of 8");
  constexpr int WH = WB / 2;
  using S = Shape<D, WH, 0>;
  constexpr int NWH = S::NW;                 // words of one half-entry (D * WH)
  extern __shared__ __align__(16) uint32_t smem[];
  __shared__ int s_chunk;
  const int half = threadIdx.x & 1;
  const unsigned pair = 3u << (threadIdx.x & 30);
  int loaded = -1;
  uint32_t H[S::NR * WH];
  for (;;) {
    if (threadIdx.x == 0) s_chunk = (int)atomicAdd(args.head, 1u);
    __syncthreads();
    const int c = s_chunk;
    __syncthreads();
    if (c >= args.nchunks) break;
    const BatchChunk ch = args.chunks[c];
    const BatchProblem pr = args.problems[ch.problem];
    const int R = pr.R, k = pr.k, B = pr.B, nh = R - 1 - k;
    const int head = ((R * WH + 3 * WH) + 3) & ~3;
    const int span = batch_split_span(D, WB, R, B);
    uint32_t* sA = smem + half * span;
    uint32_t* sH0 = sA + R * WH + WH;
    uint32_t* sT = sA + head;
    if (ch.problem != loaded) {
      // word w of a packed row goes to half w / WH
      for (int t = threadIdx.x; t < R * WB; t += blockDim.x) {
        const int i = t / WB, w = t - i * WB, hh = w / WH;
        smem[hh * span + i * WH + (w - hh * WH)] = pr.A[t];
      }
      for (int t = threadIdx.x; t < WB; t += blockDim.x) {
        const int hh = t / WH, w = t - hh * WH;
        uint32_t* v = smem + hh * span + R * WH;
        v[w] = pr.tot[t];
        v[WH + w] = pr.hinit[t];
        v[2 * WH + w] = pr.tbias[t];
      }
      __syncthreads();
      for (int t = threadIdx.x; t < 2 * B; t += blockDim.x) {
        const int j = t >> 1;
        uint32_t* base = smem + (t & 1) * span;
        batch_build_entry<D, WH, 0>(j, k, base, base + R * WH, base + R * WH + 2 * WH,
                                    base + head + j * NWH);
      }
      __syncthreads();
      loaded = ch.problem;
    }
    const unsigned long long WL = pr.walk_len;
    int best = INT_MIN;
    unsigned long long best_h = 0ull;
    // both threads of a pair take the same walks (same control flow)
    for (unsigned long long wk = ch.walk_begin + (threadIdx.x >> 1); wk < ch.walk_end; wk += blockDim.x >> 1) {
      if constexpr (D == 3) {   // walks holding no class minimum (table_kernel.cuh)
        if (pr.sym_digits > 0 && !walk_holds_class_min<3>(wk, pr.sym_digits, pr.sym_pw)) continue;
      }
      const unsigned long long h0 = wk * WL;
      seed_high<D, WH, 0>(H, sA, sH0, k, nh, h0);
      for (unsigned long long u = 0; u < WL; ++u) {
        if (u) {
          const unsigned long long h = h0 + u;
          int i, a, b;
          if (D <= 2) {
            i = __ffsll((long long)u) - 1;
            b = (int)(((h >> (i + 1)) & 1ull) ^ 1ull);
            a = b ^ 1;
          } else {
            unsigned long long q = u;
            i = 0;
            while (q % 3ull == 0ull) { q /= 3ull; ++i; }
            const int cc = (int)(q % 3ull);
            const int par = (int)((wk ^ (q / 3ull)) & 1ull);
            b = par ? 2 - cc : cc;
            a = par ? 3 - cc : cc - 1;
          }
          move_row<D, WH, 0>(H, sA + (k + i) * WH, a, b);
        }
        const int m = scan_max_split<D, WH>(H, sT, B, pair);
        if (m > best) { best = m; best_h = h0 + u; }
      }
    }
    long long bv = LLONG_MIN;
    unsigned long long bn = ULLONG_MAX;
    if (best != INT_MIN) {   // the pair holds the same best and best_h
      seed_high<D, WH, 0>(H, sA, sH0, k, nh, best_h);
      const bool rev = (best_h & 1ull) != 0ull;
      for (int jj = 0; jj < B; ++jj) {
        const int je = rev ? B - 1 - jj : jj;
        int v = entry_value<D, WH, 0>(H, sT + je * NWH);
        v += __shfl_xor_sync(pair, v, 1);
        if (v == best) {
          bn = best_h * (unsigned long long)B + (unsigned long long)jj;
          break;
        }
      }
      bv = (long long)best - pr.value_offset;
    }
    block_best(bv, bn);
    if (threadIdx.x == 0) { args.chunk_results[c].value = bv; args.chunk_results[c].index = bn; }
  }
}

// Fold each matrix's chunk slots [ranges[2p], ranges[2p+1]) into results[p].
// (A template so that every translation unit including this header may see
// its definition.)
template <int Unused = 0>
__global__ void batch_fold_kernel(const Slot* chunk_results, const int* ranges, int nproblems,
                                  Slot* results) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nproblems) return;
  long long v = LLONG_MIN;
  unsigned long long n = ULLONG_MAX;
  for (int c = ranges[2 * p]; c < ranges[2 * p + 1]; ++c) {
    const Slot s = chunk_results[c];
    if (better(s.value, s.index, v, n)) { v = s.value; n = s.index; }
  }
  results[p].value = v;
  results[p].index = n;
}

}  // namespace ld
