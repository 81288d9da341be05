// Kernel instances, compiled in separate translation units.
#pragma once

namespace ld {

// table_kernel<D, WB, WA> by (D, WB, WA): D in 1..10, WB int32 words (0..64),
// WA int8x4 words (0..32).  Instances:
//   D = 1: WB <= 4 with WA <= 16 (mixed), WA <= 32 with WB = 0, WB <= 64 with WA = 0
//   D = 2: WB <= 64 with WA = 0, WA <= 32 with WB = 0
//   D = 3: WB <= 64 with WA = 0, WA <= 32 with WB = 0
//   D = 4..10: WA in 1..8 with WB = 0, WB in 4, 8, 12, 16 with WA = 0
using TableKernelTab = const void* [11][65][33];
void table_register_d1_mix(TableKernelTab& t);
void table_register_d1_p8(TableKernelTab& t);
void table_register_d1_p32a(TableKernelTab& t);
void table_register_d1_p32b(TableKernelTab& t);
void table_register_d2(TableKernelTab& t);
void table_register_d3(TableKernelTab& t);
void table_register_dn(TableKernelTab& t);

// table_kernel<1, WB, WA, true> (LM, marginal column linear in word 0) by
// (WB, WA): WB in 1..2, WA in 0..16
using TableKernelLinTab = const void* [3][17];
void table_register_d1_lin(TableKernelLinTab& t);

// table_kernel<1, WB, WA, LIN, PAIR = true> by (LIN, WB, WA): WB + WA <= 10
// (LIN only with WB in 1..2)
using TableKernelPairTab = const void* [2][11][17];
void table_register_pair(TableKernelPairTab& t);
// table_kernel<D, WB, WA, false, PAIR = true> for D = 2, 3 by (D - 2, WB, WA):
// WB in 1..8 with WA = 0, or WA in 1..8 with WB = 0
using TableKernelPair23Tab = const void* [2][9][9];
void table_register_pair23(TableKernelPair23Tab& t);

// nullptr when not instantiated
const void* table_kernel_mixed_ptr(int D, int WB, int WA);
const void* table_kernel_pair_ptr(int D, int WB, int WA, int lin);
const void* table_kernel_lin_ptr(int WB, int WA);
// all columns in one lane width: PK = 1 (int32, W words) or 4 (int8x4, W words)
const void* table_kernel_ptr(int D, int W, int PK);
// pruned-search kernels {walk_bound_kernel, prune_scan_kernel} for (D, WB, WA):
//   D = 1: WB <= 2 with WA <= 16, WB in 4, 8, .., 64 with WA = 0
//   D = 2: WB in 4, 8, .., 48 (WA = 0) or WA in 4, 8, .., 32 (WB = 0)
//   D = 3: WB in 4, 8, .., 32 (WA = 0) or WA in 4, 8, .., 32 (WB = 0)
using PruneKernelTab = const void* [4][65][33][2];
void prune_register_d1(PruneKernelTab& t);
void prune_register_d23(PruneKernelTab& t);
// {nullptr, nullptr} when not instantiated
void prune_kernel_ptrs(int D, int WB, int WA, const void** bound, const void** scan);
// batch_table_kernel<D, WB, WA> for the batch lane classes (batch_inst.cu), and
// the per-matrix fold kernel
const void* batch_kernel_ptr(int D, int WB, int WA);
// column-split instance of an int32 class (WB = 40, 48, 56, 64), or null
const void* batch_split_kernel_ptr(int D, int WB);
const void* batch_fold_kernel_ptr();
// table_split_kernel<D, PK, PW, S> (split_kernel.cuh) by
// [D][PK == 4][PW / 4 - 1 (PW = 4, 8, .., 32)][S = 2, 4, 8]: the column-split
// form of the table kernel (S lanes per high index, PW words each); nullptr
// when not instantiated.  Instances: split_d1.cu, split_d2.cu, split_d3.cu,
// split_dn.cu.
using SplitKernelTab = const void* [11][2][8][3];
void split_register_d1(SplitKernelTab& t);
void split_register_d2(SplitKernelTab& t);
void split_register_d3(SplitKernelTab& t);
void split_register_d4_6(SplitKernelTab& t);
void split_register_d7_10(SplitKernelTab& t);
const void* table_split_kernel_ptr(int D, int PK, int PW, int S);
// wide_kernel<IT, PC, MULTI>, PC in {1,2,4,...,128}
// sym = 1: the instance that takes the walks passing the label-symmetry test by rank
const void* wide_kernel_ptr(int i64, int PC, int multi, int sym);

}  // namespace ld

#define LD_WIDE_MAXD 10
