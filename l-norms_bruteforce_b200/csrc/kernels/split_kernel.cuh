// Column-split form of the table kernel, for matrices wider than one
// thread's register vectors hold (d <= 3 past 64 int32 / 128 8-bit columns,
// d >= 4 past 16 int32 / 32 8-bit columns).
//
// The enumeration is the table kernel's (table_kernel.cuh): Gray index
// N = h * B + j, a shared-memory table of the low rows' partial sums for all
// B low labelings, walks over the high indices h with one row moved per
// step, the value of a labeling the sum over columns and message vectors of
// |H - T_j|.  The difference is who holds the columns: S adjacent lanes of a
// warp (a group) share one high index, and lane g holds slice g of the
// columns (PW words of every message vector, all in 32-bit lanes or all in
// four 8-bit lanes per word).  Each slice has its own region of shared
// memory (its words of the rows, totals, initial H, table bias and table),
// laid out as a table-kernel problem of width PW, so the table kernel's
// helpers run on a slice unchanged.
//
// Values of S entries at a time.  A lane forms its slice's partial sums for
// the S entries of a tile, entry (g + r) mod S into acc[r], r = 0 .. S-1, as
// S independent accumulator chains; then a ring reduce-scatter of S - 1
// steps (one shuffle and one add per step, with register indices fixed at
// compile time) leaves in acc[0] of lane g the full value of entry g of the
// tile.  Per labeling this costs (2S - 1) / S instructions on top of the
// absolute-difference-accumulates, against log2(S) shuffles and adds for a
// reduction of each entry on its own.  The table has Bp entries, B rounded
// up to a multiple of S; the extra ones repeat entry 0, which changes no
// maximum.  Ties: each lane keeps the smallest h attaining its maximum, the
// group agrees on the smallest h at the group's maximum, and rescans that
// block for the smallest Gray position, as in the table kernel.
#pragma once
#include "batch_kernel.cuh"
#include "table_kernel.cuh"

namespace ld {

struct SplitArgs {
  TableArgs t;   // image (full-width rows), geometry, label symmetry, reduction
  int W;         // words of a packed row: S * PW
  int Bp;        // table entries: B rounded up to a multiple of S
  int span;      // words of one slice's shared-memory region (bank padding included)
};

// words of one slice region before padding: rows, totals, initial H, table
// bias (PW words each, rounded up to 16 bytes), then Bp entries of D x PW
__host__ __device__ inline int split_region_words(int D, int PW, int R, int Bp) {
  return ((R * PW + 3 * PW + 3) & ~3) + Bp * D * PW;
}

// Table entry j of one slice (PW words per vector) into e.
template <int D, int SB, int SA>
__device__ __forceinline__ void split_build_entry(int j, int k, const uint32_t* sA, const uint32_t* sTot,
                                                  const uint32_t* sTb, uint32_t* e) {
  if constexpr (D >= 4) build_entry_dn<D, SB, SA>(j, sA, sTot, e, k);
  else batch_build_entry<D, SB, SA>(j, k, sA, sTot, sTb, e);
}

// Full value of entry j0 + g (j0 a multiple of S) for lane g of a group:
// its slice's partial sums of the tile's S entries, then the ring
// reduce-scatter with the group's lanes (src = the lane before, mod S).
template <int D, int SB, int SA, int S>
__device__ __forceinline__ int split_tile(const uint32_t* H, const uint32_t* sT, int j0, int g, unsigned gmask,
                                          int src) {
  using Sh = Shape<D, SB, SA>;
  uint32_t acc[S];
#pragma unroll
  for (int r = 0; r < S; ++r) {
    const uint4* t = reinterpret_cast<const uint4*>(sT + (j0 + ((g + r) & (S - 1))) * Sh::NW);
    uint32_t a0 = 0u, a1 = 0u;
#pragma unroll
    for (int q = 0; q < Sh::NW / 4; ++q) sad4<D, SB, SA>(H, t[q], q, a0, a1);
    acc[r] = a0 + a1;
  }
  // step t: acc[S-1-t] (this lane's partial of entry g + S-1-t) gains the
  // running sum of that entry from the lane before; after S - 1 steps
  // acc[0] holds all S slices of entry g
#pragma unroll
  for (int t = 1; t < S; ++t) acc[S - 1 - t] += __shfl_sync(gmask, acc[S - t], src, S);
  return (int)acc[0];
}

// Two tiles at once (entries j0 .. j0 + 2S - 1): 2S independent partial
// sums, then the two rings interleaved, so that each shuffle's latency is
// hidden behind the other ring's step.  v0 / v1: entry j0 + g / j0 + S + g.
template <int D, int SB, int SA, int S>
__device__ __forceinline__ void split_tile2(const uint32_t* H, const uint32_t* sT, int j0, int g, unsigned gmask,
                                            int src, int& v0, int& v1) {
  using Sh = Shape<D, SB, SA>;
  uint32_t acc[S], acd[S];
#pragma unroll
  for (int r = 0; r < S; ++r) {
    const int e = (g + r) & (S - 1);
    const uint4* t0 = reinterpret_cast<const uint4*>(sT + (j0 + e) * Sh::NW);
    const uint4* t1 = reinterpret_cast<const uint4*>(sT + (j0 + S + e) * Sh::NW);
    uint32_t a0 = 0u, a1 = 0u, b0 = 0u, b1 = 0u;
#pragma unroll
    for (int q = 0; q < Sh::NW / 4; ++q) {
      sad4<D, SB, SA>(H, t0[q], q, a0, a1);
      sad4<D, SB, SA>(H, t1[q], q, b0, b1);
    }
    acc[r] = a0 + a1;
    acd[r] = b0 + b1;
  }
#pragma unroll
  for (int t = 1; t < S; ++t) {
    const uint32_t x = __shfl_sync(gmask, acc[S - t], src, S);
    const uint32_t y = __shfl_sync(gmask, acd[S - t], src, S);
    acc[S - 1 - t] += x;
    acd[S - 1 - t] += y;
  }
  v0 = (int)acc[0];
  v1 = (int)acd[0];
}

// max over the Bp table entries: pairs of tiles, then a last single tile
template <int D, int SB, int SA, int S>
__device__ __forceinline__ int split_scan(const uint32_t* H, const uint32_t* sT, int Bp, int g, unsigned gmask,
                                          int src) {
  int m = INT_MIN;
  int j0 = 0;
  for (; j0 + 2 * S <= Bp; j0 += 2 * S) {
    int v0, v1;
    split_tile2<D, SB, SA, S>(H, sT, j0, g, gmask, src, v0, v1);
    m = max(m, max(v0, v1));
  }
  if (j0 < Bp) m = max(m, split_tile<D, SB, SA, S>(H, sT, j0, g, gmask, src));
  return m;
}

// Two high indices per group (K = 2): a tile's slice of each entry is read
// from shared memory once and compared with both register vectors H and G.
// Each lane needs its own 16 bytes per four absolute-difference-accumulates
// (the S lanes of a group read different slices, so the read is not a
// broadcast as in the table kernel), which at one high index per lane asks
// twice what shared memory delivers (128 bytes per clock per SM) at the
// integer pipe's rate; two halve it.  mh / mg: the maxima for H and G.
template <int D, int SB, int SA, int S>
__device__ __forceinline__ void split_scan2(const uint32_t* H, const uint32_t* G, const uint32_t* sT, int Bp, int g,
                                            unsigned gmask, int src, int& mh, int& mg) {
  using Sh = Shape<D, SB, SA>;
  int m0 = INT_MIN, m1 = INT_MIN;
  for (int j0 = 0; j0 < Bp; j0 += S) {
    uint32_t acc[S], acg[S];
#pragma unroll
    for (int r = 0; r < S; ++r) {
      const uint4* t = reinterpret_cast<const uint4*>(sT + (j0 + ((g + r) & (S - 1))) * Sh::NW);
      uint32_t a0 = 0u, a1 = 0u, b0 = 0u, b1 = 0u;
#pragma unroll
      for (int q = 0; q < Sh::NW / 4; ++q) {
        const uint4 x = t[q];
        sad4<D, SB, SA>(H, x, q, a0, a1);
        sad4<D, SB, SA>(G, x, q, b0, b1);
      }
      acc[r] = a0 + a1;
      acg[r] = b0 + b1;
    }
#pragma unroll
    for (int t = 1; t < S; ++t) {
      const uint32_t x = __shfl_sync(gmask, acc[S - t], src, S);
      const uint32_t y = __shfl_sync(gmask, acg[S - t], src, S);
      acc[S - 1 - t] += x;
      acg[S - 1 - t] += y;
    }
    m0 = max(m0, (int)acc[0]);
    m1 = max(m1, (int)acg[0]);
  }
  mh = m0;
  mg = m1;
}

template <int D, int PK, int PW, int S, int K = 1>
__global__ void __launch_bounds__(kTableThreads) table_split_kernel(const SplitArgs sa) {
  static_assert(PK == 1 || PK == 4, "32-bit lanes or four 8-bit lanes per word");
  static_assert(PW % 4 == 0 && (S == 2 || S == 4 || S == 8), "slices of whole 16-byte words, 2-8 lanes");
  static_assert(K == 1 || (K == 2 && D <= 2), "two high indices per group: d <= 2 (one register vector each)");
  constexpr int SB = PK == 1 ? PW : 0, SA = PK == 4 ? PW : 0;
  using Sh = Shape<D, SB, SA>;   // one slice: WV = WT = PW
  constexpr int NW = Sh::NW;     // words of a slice entry (D * PW)
  const TableArgs& args = sa.t;
  extern __shared__ __align__(16) uint32_t smem[];
  const int R = args.R, k = args.k, B = args.B, Bp = sa.Bp, W = sa.W, span = sa.span;
  const int nh = R - 1 - k;
  const int head = (R * PW + 3 * PW + 3) & ~3;
  const int g = threadIdx.x & (S - 1);
  const unsigned gmask = ((1u << S) - 1u) << ((threadIdx.x & 31) & ~(S - 1));
  const int src = (g + S - 1) & (S - 1);
  uint32_t* sA = smem + g * span;
  uint32_t* sH0 = sA + R * PW + PW;
  uint32_t* sT = sA + head;

  // stage: word w of a packed row, total or initial vector goes to slice w / PW
  for (int t = threadIdx.x; t < R * W; t += blockDim.x) {
    const int i = t / W, w = t - i * W, r = w / PW;
    smem[r * span + i * PW + (w - r * PW)] = args.A[t];
  }
  for (int t = threadIdx.x; t < W; t += blockDim.x) {
    const int r = t / PW, w = t - r * PW;
    uint32_t* v = smem + r * span + R * PW;
    v[w] = args.tot[t];
    v[PW + w] = args.hinit[t];
    v[2 * PW + w] = args.tbias ? args.tbias[t] : 0u;
  }
  __syncthreads();
  // the table, one (entry, slice) per thread; entries B .. Bp-1 repeat entry 0
  for (int t = threadIdx.x; t < Bp * S; t += blockDim.x) {
    const int j = t / S, r = t - j * S;
    uint32_t* rb = smem + r * span;
    split_build_entry<D, SB, SA>(j < B ? j : 0, k, rb, rb + R * PW, rb + R * PW + 2 * PW, rb + head + j * NW);
  }
  __syncthreads();

  const unsigned long long G = ((unsigned long long)gridDim.x * blockDim.x) / S;   // groups
  const unsigned long long gid = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) / S;
  const unsigned long long WL = args.walk_len;
  uint32_t H[Sh::NR * PW];
  int best = INT_MIN;
  unsigned long long best_h = 0ull;
  // d >= 3 with label symmetry: the passing walks, handed out by rank; all
  // lanes of a group take the same walks (same control flow for the shuffles)
  const bool by_rank = D >= 3 && args.sym_digits > 0;
  const unsigned long long it_end = by_rank ? args.rank_end : args.walk_end;
  if constexpr (K == 2) {
    // walks it and it + G in lockstep: the same row moves at each step (the
    // step depends on the offset only); a lone last walk runs twice
    uint32_t G2[Sh::NR * PW];
    for (unsigned long long it = args.walk_begin + gid; it < it_end; it += 2 * G) {
      const unsigned long long wk = it, wg = it + G < it_end ? it + G : it;
      const unsigned long long h0 = wk * WL, g0 = wg * WL;
      seed_high<D, SB, SA>(H, sA, sH0, k, nh, h0);
      seed_high<D, SB, SA>(G2, sA, sH0, k, nh, g0);
      for (unsigned long long u = 0; u < WL; ++u) {
        if (u) {
          int i, a, b, i2, a2, b2;
          high_step<D>(wk, h0 + u, u, i, a, b);
          high_step<D>(wg, g0 + u, u, i2, a2, b2);
          move_row<D, SB, SA>(H, sA + (k + i) * PW, a, b);
          move_row<D, SB, SA>(G2, sA + (k + i2) * PW, a2, b2);
        }
        int mh, mg;
        split_scan2<D, SB, SA, S>(H, G2, sT, Bp, g, gmask, src, mh, mg);
        if (mh > best || (mh == best && h0 + u < best_h)) { best = mh; best_h = h0 + u; }
        if (mg > best || (mg == best && g0 + u < best_h)) { best = mg; best_h = g0 + u; }
      }
    }
  } else {
  for (unsigned long long it = (by_rank ? args.rank_begin : args.walk_begin) + gid; it < it_end; it += G) {
    unsigned long long wk = it;
    if constexpr (D >= 3) {
      if (by_rank) wk = walk_of_rank<D>(it, args.sym_digits, args.sym_table);
    }
    const unsigned long long h0 = wk * WL;
    seed_high<D, SB, SA>(H, sA, sH0, k, nh, h0);
    for (unsigned long long u = 0; u < WL; ++u) {
      if (u) {
        int i, a, b;
        high_step<D>(wk, h0 + u, u, i, a, b);
        move_row<D, SB, SA>(H, sA + (k + i) * PW, a, b);
      }
      const int m = split_scan<D, SB, SA, S>(H, sT, Bp, g, gmask, src);
      if (m > best) { best = m; best_h = h0 + u; }
    }
  }
  }

  // the group's maximum and the smallest high index attaining it
#pragma unroll
  for (int off = 1; off < S; off <<= 1) {
    const int ob = __shfl_xor_sync(gmask, best, off, S);
    const unsigned long long oh = __shfl_xor_sync(gmask, best_h, off, S);
    if (ob > best || (ob == best && oh < best_h)) { best = ob; best_h = oh; }
  }
  // the first index attaining it: rescan that block (every lane of the
  // group takes part), the smallest Gray position among the entries at the
  // maximum
  long long bv = LLONG_MIN;
  unsigned long long bn = ULLONG_MAX;
  if (best != INT_MIN) {
    seed_high<D, SB, SA>(H, sA, sH0, k, nh, best_h);
    const int p0 = (int)(best_h & 1ull);
    int jbest = INT_MAX;
    for (int j0 = 0; j0 < Bp; j0 += S) {
      const int v = split_tile<D, SB, SA, S>(H, sT, j0, g, gmask, src);
      const int je = j0 + g;
      if (je < B && v == best) {
        int jj;
        if constexpr (D >= 4) jj = block_pos_of_entry<D>(je, k, p0);
        else jj = p0 ? B - 1 - je : je;   // d <= 3: the low word is read backwards for odd h
        jbest = min(jbest, jj);
      }
    }
#pragma unroll
    for (int off = 1; off < S; off <<= 1) jbest = min(jbest, __shfl_xor_sync(gmask, jbest, off, S));
    if (jbest != INT_MAX) bn = best_h * (unsigned long long)B + (unsigned long long)jbest;
    bv = (long long)best - args.value_offset;
  }
  grid_reduce(bv, bn, args.red);
}

}  // namespace ld
