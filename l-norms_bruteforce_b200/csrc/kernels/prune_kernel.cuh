// Pruned exact search: the table kernel's enumeration with integer upper
// bounds that skip whole blocks of labelings which cannot beat an incumbent.
//
// Split the free rows into top rows (the Gray digits of a walk index), walk
// rows (the fw digits a thread walks) and low rows (the tabulated k digits).
// For any labeling, per message m and column l the column sum is
// P_ml + Q_ml, P over the fixed and top rows, Q over the rest, so
//     value <= sum_ml |P_ml| + max over the rest's labelings of sum_ml |Q_ml|
// and the second term is exactly the L_d norm (for LM: the marginal norm)
// of the rest rows alone, computed beforehand by the plain solver.  The
// search runs in two launches:
//   1. walk_bound_kernel: for every walk, the bound with P over the top rows
//      and the rest = walk + low rows; walks whose bound is below the
//      incumbent are dropped, the others are appended to a list;
//   2. prune_scan_kernel: every listed walk is walked as in the table kernel;
//      for every high index h the bound with P = H(h) and the rest = the low
//      rows decides whether its B labelings need evaluating, and the
//      surviving h are evaluated by the whole warp together (H broadcast by
//      shuffles, the B table entries split over the lanes).
// Only bounds strictly below the incumbent prune, so every labeling that
// attains the maximum is evaluated and the smallest Gray index among them is
// the one reported: the result equals the plain enumeration's.
//
// Bounds are formed in the kernel's representation: for d = 1 the register
// vector is the signed sum (for LM with column 0 shifted by K_H >= 0, so its
// absolute value is the shifted signed sum); for d = 2 the messages are H
// and T - H, for d = 3 H1, H2 and T - H1 - H2, where T is the column total of
// the rows in P (uploaded per level).
#pragma once
#include "table_kernel.cuh"

namespace ld {

struct PruneArgs {
  TableArgs t;                    // the table kernel's operands (walk range = all walks)
  const uint32_t* ttop;           // WT words: column totals of the fixed + top rows (d >= 2)
  const uint32_t* thigh;          // WT words: column totals of the fixed + top + walk rows (d >= 2)
  long long threshold;            // incumbent, in the kernel's value representation
  long long m_walk;               // norm of the walk + low rows (representation-adjusted)
  long long m_low;                // norm of the low rows (representation-adjusted)
  unsigned long long* list;       // surviving walk indices
  unsigned long long* list_count; // number of surviving walks
  unsigned long long* stats;      // [0] walks kept, [1] h kept, [2] h visited
};

constexpr int kPruneThreads = 128;

// sum over the register vectors' lanes of |x| for d = 1, or of the message
// vectors' |.| for d = 2, 3 (T = column totals of the rows the vectors cover)
template <int D, int WB, int WA>
__device__ __forceinline__ long long prefix_abs(const uint32_t* H, const uint32_t* T) {
  using S = Shape<D, WB, WA>;
  static_assert(D != 3 || S::NR == 3, "pruned d = 3 shapes keep H1 + H2 in registers");
  uint32_t acc = 0u;
  if (D == 1) {
#pragma unroll
    for (int w = 0; w < S::WV; ++w) acc = wsad<WB>(w, H[w], 0u, acc);
  } else if (D == 2) {
#pragma unroll
    for (int w = 0; w < S::WV; ++w) {
      acc = wsad<WB>(w, H[w], 0u, acc);
      acc = wsad<WB>(w, H[w], T[w], acc);
    }
  } else {
#pragma unroll
    for (int w = 0; w < S::WV; ++w) {
      acc = wsad<WB>(w, H[w], 0u, acc);
      acc = wsad<WB>(w, H[S::WV + w], 0u, acc);
      acc = wsad<WB>(w, H[2 * S::WV + w], T[w], acc);
    }
  }
  return (long long)acc;
}

// H over the fixed row and the top rows only (digits fw.. of the high index)
template <int D, int WB, int WA>
__device__ __forceinline__ void seed_top(uint32_t* H, const uint32_t* sA, const uint32_t* sH0,
                                         int k, int fw, int nh, unsigned long long h) {
  using S = Shape<D, WB, WA>;
#pragma unroll
  for (int w = 0; w < S::WV; ++w) H[w] = sH0[w];
#pragma unroll
  for (int v = 1; v < S::NR; ++v)
#pragma unroll
    for (int w = 0; w < S::WV; ++w) H[v * S::WV + w] = 0u;
  if (D <= 2) {
    const unsigned long long g = h ^ (h >> 1);
    for (int t = fw; t < nh; ++t) {
      const int lab = (int)((g >> t) & 1ull);
      const uint32_t* row = sA + (k + t) * S::WT;
      if (D == 1) { if (lab) add_row<D, WB, WA>(H, row, 0); else sub_row<D, WB, WA>(H, row, 0); }
      else if (lab) add_row<D, WB, WA>(H, row, 0);
    }
  } else {
    unsigned long long q = h;
    for (int t = 0; t < fw; ++t) q /= 3ull;
    for (int t = fw; t < nh; ++t) {
      const int r = (int)(q % 6ull);
      const int lab = r < 3 ? r : 5 - r;
      q /= 3ull;
      const uint32_t* row = sA + (k + t) * S::WT;
      if (lab == 1) { add_row<D, WB, WA>(H, row, 0); if (S::NR == 3) add_row<D, WB, WA>(H, row, 2); }
      else if (lab == 2) { add_row<D, WB, WA>(H, row, 1); if (S::NR == 3) add_row<D, WB, WA>(H, row, 2); }
    }
  }
}

// add the walk rows (digits 0..fw-1) of high index h to a top-row vector
template <int D, int WB, int WA>
__device__ __forceinline__ void add_walk_rows(uint32_t* H, const uint32_t* sA, int k, int fw,
                                              unsigned long long h) {
  using S = Shape<D, WB, WA>;
  if (D <= 2) {
    const unsigned long long g = h ^ (h >> 1);
    for (int t = 0; t < fw; ++t) {
      const int lab = (int)((g >> t) & 1ull);
      const uint32_t* row = sA + (k + t) * S::WT;
      if (D == 1) { if (lab) add_row<D, WB, WA>(H, row, 0); else sub_row<D, WB, WA>(H, row, 0); }
      else if (lab) add_row<D, WB, WA>(H, row, 0);
    }
  } else {
    unsigned long long q = h;
    for (int t = 0; t < fw; ++t) {
      const int r = (int)(q % 6ull);
      const int lab = r < 3 ? r : 5 - r;
      q /= 3ull;
      const uint32_t* row = sA + (k + t) * S::WT;
      if (lab == 1) { add_row<D, WB, WA>(H, row, 0); if (S::NR == 3) add_row<D, WB, WA>(H, row, 2); }
      else if (lab == 2) { add_row<D, WB, WA>(H, row, 1); if (S::NR == 3) add_row<D, WB, WA>(H, row, 2); }
    }
  }
}

// stage rows, vectors and (for the scan) the table into shared memory
template <int D, int WB, int WA>
__device__ __forceinline__ void stage(const PruneArgs& args, uint32_t* smem, bool with_table) {
  using S = Shape<D, WB, WA>;
  constexpr int WT = S::WT;
  const TableArgs& ta = args.t;
  const int R = ta.R;
  uint32_t* sA = smem;
  uint32_t* sTot = sA + R * WT;
  uint32_t* sH0 = sTot + WT;
  uint32_t* sTb = sH0 + WT;
  uint32_t* sTtop = sTb + WT;
  uint32_t* sThigh = sTtop + WT;
  for (int t = threadIdx.x; t < R * WT; t += blockDim.x) sA[t] = ta.A[t];
  for (int t = threadIdx.x; t < WT; t += blockDim.x) {
    sTot[t] = ta.tot[t];
    sH0[t] = ta.hinit[t];
    sTb[t] = ta.tbias ? ta.tbias[t] : 0u;
    sTtop[t] = args.ttop[t];
    sThigh[t] = args.thigh[t];
  }
  __syncthreads();
  if (!with_table) return;
  uint32_t* sT = smem + (((R * WT + 5 * WT) + 3) & ~3);
  const int k = ta.k, B = ta.B;
  for (int j = threadIdx.x; j < B; j += blockDim.x) {
    uint32_t L1[S::WV], L2[S::WV];
#pragma unroll
    for (int w = 0; w < S::WV; ++w) { L1[w] = D == 1 ? sTb[w] : 0u; L2[w] = 0u; }
    if (D <= 2) {
      const unsigned g = (unsigned)j ^ ((unsigned)j >> 1);
      for (int i = 0; i < k; ++i) {
        const int lab = (g >> i) & 1u;
        const uint32_t* row = sA + i * WT;
        if (D == 1) {
#pragma unroll
          for (int w = 0; w < S::WV; ++w) L1[w] = lab ? wsub<WB>(w, L1[w], row[w]) : wadd<WB>(w, L1[w], row[w]);
        } else if (lab) {
#pragma unroll
          for (int w = 0; w < S::WV; ++w) L1[w] = wadd<WB>(w, L1[w], row[w]);
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
          for (int w = 0; w < S::WV; ++w) L1[w] = wadd<WB>(w, L1[w], row[w]);
        } else if (lab == 2) {
#pragma unroll
          for (int w = 0; w < S::WV; ++w) L2[w] = wadd<WB>(w, L2[w], row[w]);
        }
      }
    }
    uint32_t* e = sT + j * S::NW;
#pragma unroll
    for (int w = 0; w < WT; ++w) {
      if (w < S::WV) {
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
  __syncthreads();
}

__host__ __device__ inline int prune_smem_words(int D, int W, int R, int B, bool with_table) {
  int head = R * W + 5 * W;
  head = (head + 3) & ~3;
  return head + (with_table ? B * D * W : 0);
}

// Launch 1: bound every walk's top-row prefix; list the walks that survive.
// Each thread takes a contiguous run of walk indices and visits them in
// order: the top rows' labels are the reflected Gray code of the walk index
// (binary for d <= 2, 3-ary for d = 3), so consecutive walks differ in one
// top row, and the prefix vector is seeded once per run and then updated by
// one row move per walk.
template <int D, int WB, int WA>
__global__ void __launch_bounds__(kPruneThreads) walk_bound_kernel(const PruneArgs args) {
  using S = Shape<D, WB, WA>;
  extern __shared__ __align__(16) uint32_t smem[];
  stage<D, WB, WA>(args, smem, false);
  const TableArgs& ta = args.t;
  const int R = ta.R, k = ta.k, fw = ta.fw, nh = R - 1 - k;
  const uint32_t* sA = smem;
  const uint32_t* sH0 = smem + R * S::WT + S::WT;
  const uint32_t* sTtop = smem + R * S::WT + 3 * S::WT;
  const unsigned long long T = (unsigned long long)gridDim.x * blockDim.x;
  const unsigned long long tid = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  unsigned long long kept = 0;
  // every lane of a warp runs the same number of iterations (ballots below)
  const unsigned long long nw = ta.walk_end - ta.walk_begin;
  const unsigned long long run = (nw + T - 1) / T;
  const unsigned long long first = ta.walk_begin + tid * run;
  uint32_t H[S::NR * S::WV];
  // d = 3 with label symmetry: a walk that holds no smallest index of a
  // class (walk_holds_class_min, table_kernel.cuh) is dropped as well
  const int P = D == 3 ? ta.sym_digits : 0;
  unsigned long long pw = 1ull;
  for (int t = 1; t < P; ++t) pw *= 3ull;
  for (unsigned long long r = 0; r < run; ++r) {
    const unsigned long long wk = first + r;
    bool keep = false;
    if (wk < ta.walk_end) {
      if (r == 0) {
        seed_top<D, WB, WA>(H, sA, sH0, k, fw, nh, wk * ta.walk_len);
      } else {
        // the one top row whose label differs between walks wk - 1 and wk
        int i, a, b;
        if (D <= 2) {
          i = __ffsll((long long)wk) - 1;
          b = (int)(((wk >> (i + 1)) & 1ull) ^ 1ull);
          a = b ^ 1;
        } else {
          unsigned long long q = wk;
          i = 0;
          while (q % 3ull == 0ull) { q /= 3ull; ++i; }
          const int c = (int)(q % 3ull);
          const int par = (int)((q / 3ull) & 1ull);
          b = par ? 2 - c : c;
          a = par ? 3 - c : c - 1;
        }
        move_row<D, WB, WA>(H, sA + (k + fw + i) * S::WT, a, b);
      }
      keep = prefix_abs<D, WB, WA>(H, sTtop) + args.m_walk >= args.threshold;
      if constexpr (D == 3) {
        if (P > 0 && keep) keep = walk_holds_class_min<3>(wk, P, pw);
      }
    }
    const unsigned mask = __ballot_sync(0xffffffffu, keep);
    if (mask) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(args.list_count, (unsigned long long)__popc(mask));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (keep) args.list[base + __popc(mask & ((1u << lane) - 1u))] = wk;
    }
    kept += keep ? 1ull : 0ull;
  }
  if (kept) atomicAdd(&args.stats[0], kept);
}

// Launch 2: walk the listed walks; bound each high index; evaluate the
// surviving ones with the whole warp.
template <int D, int WB, int WA>
__global__ void __launch_bounds__(kPruneThreads) prune_scan_kernel(const PruneArgs args) {
  using S = Shape<D, WB, WA>;
  constexpr int WT = S::WT, NW = S::NW, NREG = S::NR * S::WV;
  extern __shared__ __align__(16) uint32_t smem[];
  stage<D, WB, WA>(args, smem, true);
  const TableArgs& ta = args.t;
  const int R = ta.R, k = ta.k, B = ta.B, fw = ta.fw, nh = R - 1 - k;
  const uint32_t* sA = smem;
  const uint32_t* sH0 = smem + R * WT + WT;
  const uint32_t* sThigh = smem + R * WT + 4 * WT;
  const uint32_t* sT = smem + (((R * WT + 5 * WT) + 3) & ~3);
  const unsigned long long T = (unsigned long long)gridDim.x * blockDim.x;
  const unsigned long long tid = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const unsigned long long WL = ta.walk_len;
  const unsigned long long nlist = *args.list_count;
  // Few surviving walks would leave most threads idle, so each walk is cut
  // into `split` parts of PL consecutive high indices (at least 8 each), one
  // part per thread; every part is seeded directly and then walked.
  unsigned long long split = nlist ? T / nlist : 1ull;
  const unsigned long long max_split = WL >= 16ull ? WL / 8ull : 1ull;
  split = split < 1ull ? 1ull : (split > max_split ? max_split : split);
  const unsigned long long PL = (WL + split - 1) / split;
  const unsigned long long items = nlist * split;
  const unsigned long long rounds = (items + T - 1) / T;
  long long bv = LLONG_MIN;
  unsigned long long bn = ULLONG_MAX;
  unsigned long long hk = 0, hv = 0;
  uint32_t H[NREG];
  for (unsigned long long r = 0; r < rounds; ++r) {
    const unsigned long long item = tid + r * T;
    const unsigned long long slot = item / split, part = item % split;
    const unsigned long long u0 = part * PL;
    const bool live = item < items && u0 < WL;
    const unsigned long long wk = live ? args.list[slot] : 0ull;
    const unsigned long long h0 = wk * WL;
    const unsigned long long u1 = live ? (u0 + PL < WL ? u0 + PL : WL) : 0ull;
    if (live) {
      seed_top<D, WB, WA>(H, sA, sH0, k, fw, nh, h0);
      add_walk_rows<D, WB, WA>(H, sA, k, fw, h0 + u0);
    }
    for (unsigned long long uu = 0; uu < PL; ++uu) {
      const unsigned long long u = u0 + uu;
      const bool on = live && u < u1;
      const unsigned long long h = h0 + u;
      if (on && uu) {
        int i, a, b;
        if (D <= 2) {
          i = __ffsll((long long)u) - 1;
          b = (int)(((h >> (i + 1)) & 1ull) ^ 1ull);
          a = b ^ 1;
        } else {
          unsigned long long q = u;
          i = 0;
          while (q % 3ull == 0ull) { q /= 3ull; ++i; }
          const int c = (int)(q % 3ull);
          const int par = (int)((wk ^ (q / 3ull)) & 1ull);
          b = par ? 2 - c : c;
          a = par ? 3 - c : c - 1;
        }
        move_row<D, WB, WA>(H, sA + (k + i) * WT, a, b);
      }
      const bool scan = on && prefix_abs<D, WB, WA>(H, sThigh) + args.m_low >= args.threshold;
      hv += on ? 1ull : 0ull;
      hk += scan ? 1ull : 0ull;
      unsigned mask = __ballot_sync(0xffffffffu, scan);
      while (mask) {
        const int src = __ffs(mask) - 1;
        mask &= mask - 1u;
        uint32_t Hs[NREG];
#pragma unroll
        for (int w = 0; w < NREG; ++w) Hs[w] = __shfl_sync(0xffffffffu, H[w], src);
        const unsigned long long hs = __shfl_sync(0xffffffffu, h, src);
        const bool rev = (hs & 1ull) != 0ull;
        int lv = INT_MIN, ljj = INT_MAX;
        for (int jj = lane; jj < B; jj += 32) {
          const int je = rev ? B - 1 - jj : jj;
          const int v = entry_value<D, WB, WA>(Hs, sT + je * NW);
          if (v > lv) { lv = v; ljj = jj; }
        }
        // warp max of the value, then the smallest position attaining it
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          const int ov = __shfl_xor_sync(0xffffffffu, lv, off);
          const int oj = __shfl_xor_sync(0xffffffffu, ljj, off);
          if (ov > lv || (ov == lv && oj < ljj)) { lv = ov; ljj = oj; }
        }
        if (lane == src) {
          const long long v = (long long)lv - ta.value_offset;
          const unsigned long long n = hs * (unsigned long long)B + (unsigned long long)ljj;
          if (better(v, n, bv, bn)) { bv = v; bn = n; }
        }
      }
    }
  }
  if (hk) atomicAdd(&args.stats[1], hk);
  if (hv) atomicAdd(&args.stats[2], hv);
  grid_reduce(bv, bn, ta.red);
}

}  // namespace ld
