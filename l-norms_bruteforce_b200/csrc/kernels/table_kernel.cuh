// Table enumeration kernel for L_1, LM (d = 1), L_2 and L_3.
//
// The Gray index of a labeling is split as N = h * B + j, B = d^k: the k
// lowest free rows ("low rows", digits of j) and the rest ("high rows",
// digits of h).  For the d-ary reflected Gray code used by the reference
// (binary for d <= 2, L_CUDA.cu:61-63; pattern 0..d-1,d-1..0 for d >= 3,
// L_CUDA.cu:204-206), the high rows' labels are the Gray word of h and the
// low rows' labels are the Gray word of j, read backwards (B-1-j) when h is
// odd.  So every block of B consecutive indices visits all B low labelings.
//
// Each block tabulates, once, the low rows' contribution to the message
// column sums for all B low labelings (Gray order, shared memory).  Each
// thread keeps the high rows' column sums H in registers, walks h in Gray
// order (one row changes per step: one add or subtract of a row staged in
// shared memory), and for every h evaluates all B labelings as
//     sum over table vectors and columns of |H - T_j|
// with one absolute-difference-accumulate instruction per column word
// against the tabulated entry (a warp-uniform broadcast read).
//
// Column words.  A vector has WB words holding one column each as a 32-bit
// lane (`__sad`), then WA words holding four columns each as signed 8-bit
// lanes (`vabsdiff4`, the same issue cost as one `__sad`).  The host puts a
// column in an 8-bit lane only when every value either operand can take
// fits in 8 bits (the instruction forms |a - b| at full width), so the lane
// arithmetic is exact.  Rows and table vectors are padded to WT words, a
// multiple of 4, for 16-byte shared-memory loads.
//
// Message vectors per labeling (D):
//   D = 1 (L_1 / LM): s = A_fixed + sum s_i A_i;          table: tb - L
//   D = 2 (L_2):      s1 = rows labelled 1, s0 = T - s1;   table: -L1, T-L1
//     both table vectors are compared against the same register vector H
//     (|H + L1| + |H - (T - L1)|);
//   D = 3 (L_3):      s1, s2, s0 = T - s1 - s2;            table: -L1, -L2, T-L1-L2
//     with registers H1, H2 and H1+H2 (above 32 words per vector H1+H2 is
//     formed on the fly from H1 and H2 to stay within the register file).
// LM enters as L_1 with column 0 shifted by K = sum_i |A_i0|: K_H (the
// high and fixed rows' share) is added to H's column 0 and K_L (the low
// rows' share) is subtracted through the table bias tb, so that column's
// term is its signed sum plus K; K is subtracted from the result.  When
// column 0 has a 32-bit lane of its own (word 0), the LIN instances use that
// its term needs no absolute value: the table stores its negation as the
// accumulator's starting value and H's column 0 is added once per high
// index, which saves one instruction per labeling.
#pragma once
#include "common.cuh"

namespace ld {

struct TableArgs {
  const uint32_t* A;        // R x WT packed rows; row R-1 is the fixed row
  const uint32_t* tot;      // WT words: column totals over all rows (D >= 2)
  const uint32_t* hinit;    // WT words: H before any high row (D = 1: fixed row)
  const uint32_t* tbias;    // WT words added to every D = 1 table vector, or null
  int R;                    // reduced rows
  int k;                    // low rows (tabulated)
  int B;                    // d^k
  int fw;                   // Gray digits walked per seed (walk length d^fw)
  unsigned long long walk_len;
  unsigned long long walk_begin, walk_end;  // walks of this launch
  int sym_digits;           // D >= 3: digits of the walk number read by the
                            // label symmetry (0 = evaluate every walk)
  const unsigned long long* sym_table;        // completion counts (walk_of_rank)
  unsigned long long rank_begin, rank_end;    // passing walks of this launch, by rank
  long long value_offset;   // subtracted from every value (LM shift K)
  int pack16;               // every entry value lies in [0, 65536): maxima of two
                            // values packed in one word (scan_max_p16, scan_max2_p16)
  Reduce red;
};

constexpr int kTableThreads = 128;

// padded words of one row / table vector
__host__ __device__ constexpr int table_row_words(int WB, int WA) { return (WB + WA + 3) & ~3; }

// Shared memory (32-bit words): packed rows, totals, initial H, table bias,
// then the table (16-byte aligned).  W is the padded row width.
__host__ __device__ inline int table_smem_words(int D, int W, int R, int B) {
  int head = R * W + 3 * W;
  head = (head + 3) & ~3;
  return head + B * D * W;
}

template <int D, int WB, int WA>
struct Shape {
  static constexpr int WV = WB + WA;                  // computed words per vector
  static constexpr int WT = (WV + 3) & ~3;            // padded words per vector
  static constexpr int NW = D * WT;                   // words per table entry
  // register vectors: D = 3 keeps H1, H2 and (up to 32 words) H1 + H2;
  // D >= 4 keeps H_1 .. H_{D-1} and their sum
  static constexpr int NR = D == 3 ? (WV > 32 ? 2 : 3) : (D >= 4 ? D : 1);
};

template <int WB>
__device__ __forceinline__ uint32_t wadd(int w, uint32_t a, uint32_t b) {
  return w < WB ? Lanes<1>::add(a, b) : Lanes<4>::add(a, b);
}
template <int WB>
__device__ __forceinline__ uint32_t wsub(int w, uint32_t a, uint32_t b) {
  return w < WB ? Lanes<1>::sub(a, b) : Lanes<4>::sub(a, b);
}
template <int WB>
__device__ __forceinline__ uint32_t wsad(int w, uint32_t a, uint32_t b, uint32_t c) {
  return w < WB ? Lanes<1>::sad(a, b, c) : Lanes<4>::sad(a, b, c);
}

template <int D, int WB, int WA>
__device__ __forceinline__ void add_row(uint32_t* H, const uint32_t* row, int vec) {
  constexpr int WV = Shape<D, WB, WA>::WV;
#pragma unroll
  for (int w = 0; w < WV; ++w) H[vec * WV + w] = wadd<WB>(w, H[vec * WV + w], row[w]);
}

template <int D, int WB, int WA>
__device__ __forceinline__ void sub_row(uint32_t* H, const uint32_t* row, int vec) {
  constexpr int WV = Shape<D, WB, WA>::WV;
#pragma unroll
  for (int w = 0; w < WV; ++w) H[vec * WV + w] = wsub<WB>(w, H[vec * WV + w], row[w]);
}

// Move high row r from label a to label b.
template <int D, int WB, int WA>
__device__ __forceinline__ void move_row(uint32_t* H, const uint32_t* row, int a, int b) {
  if (D == 1) {  // sign a -> b: add or subtract 2 * row (as two steps, each in range)
    if (b) { add_row<D, WB, WA>(H, row, 0); add_row<D, WB, WA>(H, row, 0); }
    else   { sub_row<D, WB, WA>(H, row, 0); sub_row<D, WB, WA>(H, row, 0); }
  } else if (D == 2) {
    if (b) add_row<D, WB, WA>(H, row, 0); else sub_row<D, WB, WA>(H, row, 0);
  } else if (D >= 4) {
    // vector v holds the rows labelled v + 1; vector D - 1 their sum (the
    // unrolled tests keep every register index a compile-time constant)
#pragma unroll
    for (int v = 0; v < D - 1; ++v) {
      if (a == v + 1) sub_row<D, WB, WA>(H, row, v);
      if (b == v + 1) add_row<D, WB, WA>(H, row, v);
    }
    if (a == 0 && b != 0) add_row<D, WB, WA>(H, row, D - 1);
    if (a != 0 && b == 0) sub_row<D, WB, WA>(H, row, D - 1);
  } else {
    if (a == 1) sub_row<D, WB, WA>(H, row, 0);
    if (a == 2) sub_row<D, WB, WA>(H, row, 1);
    if (b == 1) add_row<D, WB, WA>(H, row, 0);
    if (b == 2) add_row<D, WB, WA>(H, row, 1);
    if (Shape<D, WB, WA>::NR == 3) {
      if (a == 0 && b != 0) add_row<D, WB, WA>(H, row, 2);
      if (a != 0 && b == 0) sub_row<D, WB, WA>(H, row, 2);
    }
  }
}

// H for high index h: initial vector plus every high row at its label.
template <int D, int WB, int WA>
__device__ __forceinline__ void seed_high(uint32_t* H, const uint32_t* sA, const uint32_t* sH0,
                                          int k, int nh, unsigned long long h) {
  using S = Shape<D, WB, WA>;
#pragma unroll
  for (int w = 0; w < S::WV; ++w) H[w] = sH0[w];
#pragma unroll
  for (int v = 1; v < S::NR; ++v)
#pragma unroll
    for (int w = 0; w < S::WV; ++w) H[v * S::WV + w] = 0u;
  if (D <= 2) {
    const unsigned long long g = h ^ (h >> 1);
    for (int t = 0; t < nh; ++t) {
      const int lab = (int)((g >> t) & 1ull);
      const uint32_t* row = sA + (k + t) * S::WT;
      if (D == 1) { if (lab) add_row<D, WB, WA>(H, row, 0); else sub_row<D, WB, WA>(H, row, 0); }
      else if (lab) add_row<D, WB, WA>(H, row, 0);
    }
  } else if (D >= 4) {
    unsigned long long q = h;
    for (int t = 0; t < nh; ++t) {
      const int r = (int)(q % (2ull * D));
      const int lab = r < D ? r : 2 * D - 1 - r;
      q /= (unsigned long long)D;
      if (lab == 0) continue;
      const uint32_t* row = sA + (k + t) * S::WT;
#pragma unroll
      for (int v = 0; v < D - 1; ++v)
        if (lab == v + 1) add_row<D, WB, WA>(H, row, v);
      add_row<D, WB, WA>(H, row, D - 1);
    }
  } else {
    unsigned long long q = h;
    for (int t = 0; t < nh; ++t) {
      const int r = (int)(q % 6ull);
      const int lab = r < 3 ? r : 5 - r;
      q /= 3ull;
      const uint32_t* row = sA + (k + t) * S::WT;
      if (lab == 1) { add_row<D, WB, WA>(H, row, 0); if (S::NR == 3) add_row<D, WB, WA>(H, row, 2); }
      else if (lab == 2) { add_row<D, WB, WA>(H, row, 1); if (S::NR == 3) add_row<D, WB, WA>(H, row, 2); }
    }
  }
}

// Position j in the block of high index h (N = h * B + j) whose low rows'
// labels equal those of table entry e, for D >= 4: the inverse of the map
// from a block position to its table entry.  Entry e was tabulated with the
// labels of its own digits read alone; the block's low digits are read with
// the reflection carried down from h (odd h mirrors the top low digit).
// One pass over the digits from the top recovers e's labels (reflection pe)
// and j's digits (reflection p, starting at h & 1): a digit's label is
// mirrored when the number formed by the digits above it is odd (for even D
// the parity of the digit just above, for odd D of the digit sum).
template <int D>
__device__ __forceinline__ int block_pos_of_entry(int e, int k, int p0) {
  int pw = 1;
  for (int t = 1; t < k; ++t) pw *= D;
  int j = 0, pe = 0, p = p0, rem = e;
  for (int t = 0; t < k; ++t) {
    const int ne = rem / pw;
    rem -= ne * pw;
    const int lab = pe ? D - 1 - ne : ne;
    pe = (D % 2 == 0) ? (ne & 1) : ((pe + ne) & 1);
    const int n = p ? D - 1 - lab : lab;
    p = (D % 2 == 0) ? (n & 1) : ((p + n) & 1);
    j = j * D + n;
    pw /= D;
  }
  return j;
}

// register word compared with table word q (q in [0, NW))
template <int D, int WB, int WA>
__device__ __forceinline__ constexpr int reg_of(int q) {
  using S = Shape<D, WB, WA>;
  return (D >= 3 ? (q / S::WT) : 0) * S::WV + q % S::WT;
}
template <int D, int WB, int WA>
__device__ __forceinline__ constexpr bool computed(int q) {
  using S = Shape<D, WB, WA>;
  return q % S::WT < S::WV;
}

// acc += |H - e| over the words of x (table words 4q .. 4q+3).  LIN: word 0
// is a column that enters the value linearly (the LM marginal column, whose
// term H_0 - e_0 is never negative); its table word holds -e_0, which only
// seeds the accumulator, and H_0 is added once per high index by the caller.
template <int D, int WB, int WA, bool LIN = false>
__device__ __forceinline__ void sad4(const uint32_t* H, const uint4& x, int q, uint32_t& a0, uint32_t& a1) {
  using S = Shape<D, WB, WA>;
  static_assert(!LIN || (D == 1 && WB >= 1), "the linear column is a 32-bit word of an L_1 vector");
  const uint32_t xs[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int tq = 4 * q + c;
    if (computed<D, WB, WA>(tq)) {
      // short entries (up to 16 words): one dependent chain, whose latency the
      // two entries of a scan step and the resident warps hide, with no final
      // add; longer entries alternate two chains
      uint32_t& acc = (S::NW > 16 && (c & 1)) ? a1 : a0;
      const int w = tq % S::WT;
      if (LIN && tq == 0)
        acc += xs[c];
      else if (D == 3 && S::NR == 2 && tq / S::WT == 2)   // H1 + H2, formed on the fly
        acc = wsad<WB>(w, wadd<WB>(w, H[w], H[S::WV + w]), xs[c], acc);
      else
        acc = wsad<WB>(w, H[reg_of<D, WB, WA>(tq)], xs[c], acc);
    }
  }
}

// Value of table entry e against H.
template <int D, int WB, int WA, bool LIN = false>
__device__ __forceinline__ int entry_value(const uint32_t* H, const uint32_t* e) {
  using S = Shape<D, WB, WA>;
  const uint4* t = reinterpret_cast<const uint4*>(e);
  uint32_t a0 = 0u, a1 = 0u;
#pragma unroll
  for (int q = 0; q < S::NW / 4; ++q) sad4<D, WB, WA, LIN>(H, t[q], q, a0, a1);
  return (int)(a0 + a1 + (LIN ? H[0] : 0u));
}

// max over all B table entries
template <int D, int WB, int WA, bool LIN = false>
__device__ __forceinline__ int scan_max(const uint32_t* H, const uint32_t* sT, int B) {
  using S = Shape<D, WB, WA>;
  int m = INT_MIN;
  int j = 0;
  for (; j + 2 <= B; j += 2) {
    const uint4* t0 = reinterpret_cast<const uint4*>(sT + j * S::NW);
    const uint4* t1 = reinterpret_cast<const uint4*>(sT + (j + 1) * S::NW);
    uint32_t a0 = 0u, a1 = 0u, b0 = 0u, b1 = 0u;
#pragma unroll
    for (int q = 0; q < S::NW / 4; ++q) {
      const uint4 x = t0[q];
      const uint4 y = t1[q];
      sad4<D, WB, WA, LIN>(H, x, q, a0, a1);
      sad4<D, WB, WA, LIN>(H, y, q, b0, b1);
    }
    m = max(m, max((int)(a0 + a1), (int)(b0 + b1)));
  }
  if (LIN && j > 0) m += (int)H[0];
  if (j < B) m = max(m, entry_value<D, WB, WA, LIN>(H, sT + j * S::NW));
  return m;
}

// Packed maxima.  When every value an entry can take lies in [0, 65536)
// (the host checks sum |A| + K < 65536; all terms are absolute values, and
// the LM linear column's term is never negative), two values share one word,
// the second in the high half, formed by one multiply-add (off the integer
// ALU pipe), and one 16-bit-pair max keeps both running maxima: one ALU
// instruction per two labelings instead of two.  Entries of up to 32 words
// are one accumulator chain each (two entries, or two high indices, give the
// chains their independence); longer ones alternate two chains.

// acc (+)= |H - e| over one entry, as one chain (NW <= 32) or two
template <int D, int WB, int WA, bool LIN>
__device__ __forceinline__ uint32_t entry_acc(const uint32_t* H, const uint4* t) {
  using S = Shape<D, WB, WA>;
  uint32_t a0 = 0u, a1 = 0u;
  if constexpr (S::NW <= 32) {
#pragma unroll
    for (int q = 0; q < S::NW / 4; ++q) sad4<D, WB, WA, LIN>(H, t[q], q, a0, a0);
    return a0;
  } else {
#pragma unroll
    for (int q = 0; q < S::NW / 4; ++q) sad4<D, WB, WA, LIN>(H, t[q], q, a0, a1);
    return a0 + a1;
  }
}

// scan_max with packed maxima (TableArgs::pack16)
template <int D, int WB, int WA, bool LIN = false>
__device__ __forceinline__ int scan_max_p16(const uint32_t* H, const uint32_t* sT, int B) {
  using S = Shape<D, WB, WA>;
  uint32_t m = 0u;   // low half: even entries, high half: odd entries
  int j = 0;
  for (; j + 2 <= B; j += 2) {
    const uint32_t a = entry_acc<D, WB, WA, LIN>(H, reinterpret_cast<const uint4*>(sT + j * S::NW));
    const uint32_t b = entry_acc<D, WB, WA, LIN>(H, reinterpret_cast<const uint4*>(sT + (j + 1) * S::NW));
    m = __vmaxu2(m, b * 65536u + a);
  }
  int r = max((int)(m & 0xffffu), (int)(m >> 16));
  if (LIN) r += (int)H[0];
  if (j < B) r = max(r, entry_value<D, WB, WA, LIN>(H, sT + j * S::NW));
  return r;
}

// scan_max2 with packed maxima: H's value in the low half, G's in the high
// half of each entry's word; two entries per step
template <int D, int WB, int WA, bool LIN = false>
__device__ __forceinline__ void scan_max2_p16(const uint32_t* H, const uint32_t* G, const uint32_t* sT, int B,
                                              int& mh, int& mg) {
  using S = Shape<D, WB, WA>;
  uint32_t m = 0u;
  int j = 0;
  for (; j + 2 <= B; j += 2) {
    const uint4* t0 = reinterpret_cast<const uint4*>(sT + j * S::NW);
    const uint4* t1 = reinterpret_cast<const uint4*>(sT + (j + 1) * S::NW);
    const uint32_t a0 = entry_acc<D, WB, WA, LIN>(H, t0), b0 = entry_acc<D, WB, WA, LIN>(G, t0);
    const uint32_t a1 = entry_acc<D, WB, WA, LIN>(H, t1), b1 = entry_acc<D, WB, WA, LIN>(G, t1);
    m = __vmaxu2(m, b0 * 65536u + a0);
    m = __vmaxu2(m, b1 * 65536u + a1);
  }
  if (j < B) {
    const uint4* t0 = reinterpret_cast<const uint4*>(sT + j * S::NW);
    m = __vmaxu2(m, entry_acc<D, WB, WA, LIN>(G, t0) * 65536u + entry_acc<D, WB, WA, LIN>(H, t0));
  }
  mh = (int)(m & 0xffffu) + (LIN ? (int)H[0] : 0);
  mg = (int)(m >> 16) + (LIN ? (int)G[0] : 0);
}

// D >= 4: table entry j (reflected base-D Gray word of j over the k low
// rows) is the vectors -L_1 .. -L_{D-1} (L_m: the low rows labelled m) and
// T - (L_1 + .. + L_{D-1}), written to e.
template <int D, int WB, int WA>
__device__ __forceinline__ void build_entry_dn(int j, const uint32_t* sA, const uint32_t* sTot, uint32_t* e,
                                               int k) {
  using S = Shape<D, WB, WA>;
  constexpr int WT = S::WT, WV = S::WV;
  uint32_t L[D - 1][WV];
#pragma unroll
  for (int v = 0; v < D - 1; ++v)
#pragma unroll
    for (int w = 0; w < WV; ++w) L[v][w] = 0u;
  unsigned q = (unsigned)j;
  for (int i = 0; i < k; ++i) {
    const unsigned r = q % (2u * D);
    const int lab = r < (unsigned)D ? (int)r : 2 * D - 1 - (int)r;
    q /= (unsigned)D;
    const uint32_t* row = sA + i * WT;
#pragma unroll
    for (int v = 0; v < D - 1; ++v)
      if (lab == v + 1) {
#pragma unroll
        for (int w = 0; w < WV; ++w) L[v][w] = wadd<WB>(w, L[v][w], row[w]);
      }
  }
#pragma unroll
  for (int w = 0; w < WT; ++w) {
    if (w < WV) {
      uint32_t rest = sTot[w];
#pragma unroll
      for (int v = 0; v < D - 1; ++v) {
        e[v * WT + w] = wsub<WB>(w, 0u, L[v][w]);
        rest = wsub<WB>(w, rest, L[v][w]);
      }
      e[(D - 1) * WT + w] = rest;
    } else {
#pragma unroll
      for (int v = 0; v < D; ++v) e[v * WT + w] = 0u;
    }
  }
}

// D >= 4: every entry of the table, one thread per entry.
template <int D, int WB, int WA>
__device__ __forceinline__ void build_table_dn(const uint32_t* sA, const uint32_t* sTot, uint32_t* sT, int k, int B) {
  for (int j = threadIdx.x; j < B; j += blockDim.x)
    build_entry_dn<D, WB, WA>(j, sA, sTot, sT + j * Shape<D, WB, WA>::NW, k);
}

// PAIR instances walk two high indices per thread against each table entry
// read: L_1 / LM with at most 10 words, within 64 registers so that 8
// blocks stay resident per SM; d = 2 and 3 with at most 8 words per vector,
// within 102 registers (5 blocks).  The host uses them when a launch has at
// least two walks per thread.
template <int D, bool PAIR>
constexpr int table_min_blocks() { return PAIR ? (D == 1 ? 8 : 5) : 1; }

// max over all B table entries for two register vectors H and G (two high
// indices) at once: each entry is read from shared memory once for both.
template <int D, int WB, int WA, bool LIN = false>
__device__ __forceinline__ void scan_max2(const uint32_t* H, const uint32_t* G, const uint32_t* sT, int B,
                                          int& mh, int& mg) {
  using S = Shape<D, WB, WA>;
  int m0 = INT_MIN, m1 = INT_MIN;
  for (int j = 0; j < B; ++j) {
    const uint4* t = reinterpret_cast<const uint4*>(sT + j * S::NW);
    uint32_t a0 = 0u, a1 = 0u, b0 = 0u, b1 = 0u;
#pragma unroll
    for (int q = 0; q < S::NW / 4; ++q) {
      const uint4 x = t[q];
      sad4<D, WB, WA, LIN>(H, x, q, a0, a1);
      sad4<D, WB, WA, LIN>(G, x, q, b0, b1);
    }
    m0 = max(m0, (int)(a0 + a1));
    m1 = max(m1, (int)(b0 + b1));
  }
  if (LIN) { m0 += (int)H[0]; m1 += (int)G[0]; }   // B >= 1: the loop ran
  mh = m0;
  mg = m1;
}

// Label symmetry (D >= 3).  The fixed row has label 0 and the value is
// unchanged when labels 1..D-1 are permuted, so the smallest index attaining
// the maximum is the smallest index of its class.  Reading the walk number's
// P digits (the top high digits, fixed along the walk) from the top, the
// first appearance of each label must take the smallest digit any unseen
// label could take there: the smallest unseen label where the digit is read
// directly, the largest where it is mirrored.  Otherwise swapping the two
// labels leaves the digits above unchanged and lowers this one, i.e. lowers
// every index of the walk, and the walk holds no class minimum.  With at
// most one label unseen every continuation passes.  pw = D^(P-1).  The host
// copy of the test, and the count of the walks that pass, are in symmetry.c.
template <int D>
__device__ __forceinline__ bool walk_holds_class_min(unsigned long long wk, int P, unsigned long long pw) {
  unsigned used = 1u;   // label 0 (the fixed row's) is never moved
  int seen = 1, par = 0;
  unsigned long long rem = wk;
  for (int q = P - 1; q >= 0 && seen < D - 1; --q) {
    int n = 0;   // digit q: rem < D * pw
#pragma unroll
    for (int t = 0; t < D - 1; ++t)
      if (rem >= pw) { rem -= pw; ++n; }
    const int lab = par ? D - 1 - n : n;
    if (!((used >> lab) & 1u)) {
      const unsigned unused = ~used & ((1u << D) - 1u);
      const int want = par ? 31 - __clz((int)unused) : __ffs((int)unused) - 1;
      if (lab != want) return false;
      used |= 1u << lab;
      ++seen;
    }
    // reflection of the next digit: parity of the number formed by the
    // digits so far (odd D: of their sum; even D: of the last one)
    par = (D & 1) ? (par ^ (n & 1)) : (n & 1);
    pw /= (unsigned long long)D;
  }
  return true;
}

// The passing walk of rank i (increasing walk numbers), so that threads take
// only walks that run, evenly.  f[(used >> 1)][par][r] counts the passing
// continuations of r more digits after a prefix that has seen the labels in
// `used` and whose next digit has reflection par (built on the host by the
// digit DP of symmetry.c, which holds the host copy of this function).  Digit
// by digit from the top, the digit is the first whose passing continuations
// reach past i; once at most one label is unseen every continuation passes
// and the rest of i is the remaining digits.
template <int D>
__device__ __forceinline__ unsigned long long walk_of_rank(unsigned long long i, int P,
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

// One step of a walk of high indices h0, h0 + 1, .. (h0 = wk * walk length,
// a multiple of the walk length): from h - 1 to h (u = h - h0 > 0) high row
// i moves from label a to label b.
template <int D>
__device__ __forceinline__ void high_step(unsigned long long wk, unsigned long long h, unsigned long long u,
                                          int& i, int& a, int& b) {
  if (D <= 2) {
    i = __ffsll((long long)u) - 1;            // == ctz(h): h0 is a multiple of 2^fw
    b = (int)(((h >> (i + 1)) & 1ull) ^ 1ull);
    a = b ^ 1;
  } else if (D >= 4) {
    // digit i (the lowest nonzero base-D digit of u) steps from c - 1
    // to c; its label is mirrored when h / D^(i+1) is odd
    unsigned long long q = u;
    i = 0;
    while (q % (unsigned long long)D == 0ull) { q /= (unsigned long long)D; ++i; }
    const int c = (int)(q % (unsigned long long)D);
    unsigned long long hh = h;
    for (int t = 0; t <= i; ++t) hh /= (unsigned long long)D;
    const int par = (int)(hh & 1ull);
    b = par ? D - 1 - c : c;
    a = par ? D - c : c - 1;
  } else {
    unsigned long long q = u;
    i = 0;
    while (q % 3ull == 0ull) { q /= 3ull; ++i; }
    const int c = (int)(q % 3ull);
    // parity of h / 3^(i+1) = parity of wk (times an odd power) + u / 3^(i+1)
    const int par = (int)((wk ^ (q / 3ull)) & 1ull);
    b = par ? 2 - c : c;
    a = par ? 3 - c : c - 1;
  }
}

template <int D, int WB, int WA, bool LIN = false, bool PAIR = false>
__global__ void __launch_bounds__(kTableThreads, (table_min_blocks<D, PAIR>())) table_kernel(const TableArgs args) {
  static_assert(!PAIR || (D == 1 && WB + WA <= 10) || ((D == 2 || D == 3) && WB + WA <= 8),
                "paired walks: L_1 / LM with at most 10 words, d = 2, 3 with at most 8");
  using S = Shape<D, WB, WA>;
  constexpr int WT = S::WT, WV = S::WV, NW = S::NW;
  extern __shared__ __align__(16) uint32_t smem[];
  const int R = args.R, k = args.k, B = args.B;
  const int nh = R - 1 - k;  // high rows
  uint32_t* sA = smem;
  uint32_t* sTot = sA + R * WT;
  uint32_t* sH0 = sTot + WT;
  uint32_t* sTb = sH0 + WT;
  uint32_t* sT = smem + (((R * WT + 3 * WT) + 3) & ~3);

  for (int t = threadIdx.x; t < R * WT; t += blockDim.x) sA[t] = args.A[t];
  for (int t = threadIdx.x; t < WT; t += blockDim.x) {
    sTot[t] = args.tot[t];
    sH0[t] = args.hinit[t];
    sTb[t] = args.tbias ? args.tbias[t] : 0u;
  }
  __syncthreads();

  // Tabulate the low rows' partial sums for every low labeling j (Gray order).
  if constexpr (D >= 4) build_table_dn<D, WB, WA>(sA, sTot, sT, k, B);
  else
  for (int j = threadIdx.x; j < B; j += blockDim.x) {
    uint32_t L1[WV], L2[WV];
#pragma unroll
    for (int w = 0; w < WV; ++w) { L1[w] = D == 1 ? sTb[w] : 0u; L2[w] = 0u; }
    if (D <= 2) {
      const unsigned g = (unsigned)j ^ ((unsigned)j >> 1);
      for (int i = 0; i < k; ++i) {
        const int lab = (g >> i) & 1u;
        const uint32_t* row = sA + i * WT;
        if (D == 1) {
          // entry = tb - sum s_i A_i: subtract rows labelled +1, add rows labelled -1
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
    uint32_t* e = sT + j * NW;
#pragma unroll
    for (int w = 0; w < WT; ++w) {
      if (w < WV) {
        if (D == 1) {
          e[w] = (LIN && w == 0) ? 0u - L1[w] : L1[w];
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

  // Walk high indices: walks w, w + T, ... each covering walk_len
  // consecutive (aligned) high indices, so the changed row is warp-uniform.
  const unsigned long long T = (unsigned long long)gridDim.x * blockDim.x;
  const unsigned long long tid = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long WL = args.walk_len;
  uint32_t H[S::NR * WV];
  int best = INT_MIN;
  unsigned long long best_h = 0ull;
  // Two walks (wk and wk + T) in lockstep when there are at least two walks
  // per thread: both change the same row at each step (the step depends on
  // the offset u only), each in its own direction.
  // d >= 3 with label symmetry: the passing walks, handed out by rank
  const bool by_rank = D >= 3 && args.sym_digits > 0;
  const unsigned long long it_begin = by_rank ? args.rank_begin : args.walk_begin;
  const unsigned long long it_end = by_rank ? args.rank_end : args.walk_end;
  // Walks go to threads statically (walk it_begin + tid, then every T-th),
  // or, when the launch has a walk counter, 32 (paired: 64) at a time to a
  // warp, so that threads that finish early take more: with a few walks per
  // thread the static split leaves up to one walk (pair) per thread idle at
  // the end.  Fetched walks need not come in increasing order, so every
  // update keeps the smallest high index among equal maxima.
  const int lane = threadIdx.x & 31;
  unsigned long long fetched = 0ull;
  auto fetch = [&](unsigned long long n) -> bool {   // warp-uniform; false when no walks are left
    unsigned long long base = 0ull;
    if (lane == 0) base = atomicAdd(args.red.work, n);
    fetched = __shfl_sync(0xffffffffu, base, 0);
    return it_begin + fetched < it_end;
  };
  if constexpr (PAIR) {
    uint32_t G[S::NR * WV];
    auto run_pair = [&](unsigned long long it, unsigned long long ig) {
      unsigned long long wk = it, wg = ig;
      if constexpr (D >= 3) {
        if (by_rank) {
          wk = walk_of_rank<D>(it, args.sym_digits, args.sym_table);
          wg = walk_of_rank<D>(ig, args.sym_digits, args.sym_table);
        }
      }
      const unsigned long long h0 = wk * WL, g0 = wg * WL;
      seed_high<D, WB, WA>(H, sA, sH0, k, nh, h0);
      seed_high<D, WB, WA>(G, sA, sH0, k, nh, g0);
      for (unsigned long long u = 0; u < WL; ++u) {
        if (u) {
          // both walks move the same row (the step depends on u only), each
          // between its own labels
          int i, a, b, ig2, ag, bg;
          high_step<D>(wk, h0 + u, u, i, a, b);
          high_step<D>(wg, g0 + u, u, ig2, ag, bg);
          move_row<D, WB, WA>(H, sA + (k + i) * WT, a, b);
          move_row<D, WB, WA>(G, sA + (k + ig2) * WT, ag, bg);
        }
        int mh, mg;
        if (args.pack16) scan_max2_p16<D, WB, WA, LIN>(H, G, sT, B, mh, mg);
        else scan_max2<D, WB, WA, LIN>(H, G, sT, B, mh, mg);
        // keep the smallest high index among equal maxima
        if (mh > best || (mh == best && h0 + u < best_h)) { best = mh; best_h = h0 + u; }
        if (mg > best || (mg == best && g0 + u < best_h)) { best = mg; best_h = g0 + u; }
      }
    };
    if (args.red.work) {
      while (fetch(64ull)) {
        const unsigned long long it = it_begin + fetched + lane, ig = it + 32ull;
        if (it < it_end) run_pair(it, ig < it_end ? ig : it);   // a lone walk runs twice
      }
    } else {
      for (unsigned long long it = it_begin + tid; it < it_end; it += 2 * T)
        run_pair(it, it + T < it_end ? it + T : it);
    }
  } else {
  auto run_walk = [&](unsigned long long it) {
    unsigned long long wk = it;
    if constexpr (D >= 3) {
      if (by_rank) wk = walk_of_rank<D>(it, args.sym_digits, args.sym_table);
    }
    const unsigned long long h0 = wk * WL;
    seed_high<D, WB, WA>(H, sA, sH0, k, nh, h0);
    for (unsigned long long u = 0; u < WL; ++u) {
      if (u) {
        int i, a, b;
        high_step<D>(wk, h0 + u, u, i, a, b);
        move_row<D, WB, WA>(H, sA + (k + i) * WT, a, b);
      }
      const int m = args.pack16 ? scan_max_p16<D, WB, WA, LIN>(H, sT, B) : scan_max<D, WB, WA, LIN>(H, sT, B);
      if (m > best || (m == best && h0 + u < best_h)) { best = m; best_h = h0 + u; }
    }
  };
  if (args.red.work) {
    while (fetch(32ull)) {
      const unsigned long long it = it_begin + fetched + lane;
      if (it < it_end) run_walk(it);
    }
  } else {
    for (unsigned long long it = it_begin + tid; it < it_end; it += T) run_walk(it);
  }
  }

  // The first index attaining the thread's best: rescan its block in the
  // Gray order of the low part (reversed for odd h).
  long long bv = LLONG_MIN;
  unsigned long long bn = ULLONG_MAX;
  if (best != INT_MIN) {
    seed_high<D, WB, WA>(H, sA, sH0, k, nh, best_h);
    if constexpr (D >= 4) {
      // every entry once, in table order; an entry that attains the best
      // (rare) is mapped to its block position, and the smallest is kept
      int jbest = INT_MAX;
      const int p0 = (int)(best_h & 1ull);
      for (int je = 0; je < B; ++je)
        if (entry_value<D, WB, WA, LIN>(H, sT + je * NW) == best)
          jbest = min(jbest, block_pos_of_entry<D>(je, k, p0));
      if (jbest != INT_MAX) bn = best_h * (unsigned long long)B + (unsigned long long)jbest;
    } else {
      // d <= 3: the low word is read backwards for odd h
      const bool rev = (best_h & 1ull) != 0ull;
      for (int jj = 0; jj < B; ++jj) {
        const int je = rev ? B - 1 - jj : jj;
        if (entry_value<D, WB, WA, LIN>(H, sT + je * NW) == best) {
          bn = best_h * (unsigned long long)B + (unsigned long long)jj;
          break;
        }
      }
    }
    bv = (long long)best - args.value_offset;
  }
  grid_reduce(bv, bn, args.red);
}

}  // namespace ld
