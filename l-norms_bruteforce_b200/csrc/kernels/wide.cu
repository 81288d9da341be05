// wide_kernel instances and the kernel lookup.
#include "registry.h"
#include "wide_kernel.cuh"

namespace ld {

static const TableKernelTab& table_kernels() {
  static TableKernelTab tab = {};
  static bool init = [] {
    table_register_d1_mix(tab);
    table_register_d1_p8(tab);
    table_register_d1_p32a(tab);
    table_register_d1_p32b(tab);
    table_register_d2(tab);
    table_register_d3(tab);
    table_register_dn(tab);
    return true;
  }();
  (void)init;
  return tab;
}

const void* table_kernel_mixed_ptr(int D, int WB, int WA) {
  if (D < 1 || D > 10 || WB < 0 || WB > 64 || WA < 0 || WA > 32) return nullptr;
  return table_kernels()[D][WB][WA];
}

const void* table_kernel_lin_ptr(int WB, int WA) {
  static TableKernelLinTab tab = {};
  static bool init = [] {
    table_register_d1_lin(tab);
    return true;
  }();
  (void)init;
  if (WB < 1 || WB > 2 || WA < 0 || WA > 16) return nullptr;
  return tab[WB][WA];
}

const void* table_kernel_pair_ptr(int D, int WB, int WA, int lin) {
  static TableKernelPairTab tab = {};
  static TableKernelPair23Tab tab23 = {};
  static bool init = [] {
    table_register_pair(tab);
    table_register_pair23(tab23);
    return true;
  }();
  (void)init;
  if (D == 2 || D == 3) {
    if (lin || WB < 0 || WB > 8 || WA < 0 || WA > 8) return nullptr;
    return tab23[D - 2][WB][WA];
  }
  if (D != 1 || WB < 0 || WB > 10 || WA < 0 || WA > 16 || WB + WA > 10) return nullptr;
  return tab[lin ? 1 : 0][WB][WA];
}

const void* table_kernel_ptr(int D, int W, int PK) {
  if (PK == 1) return table_kernel_mixed_ptr(D, W, 0);
  if (PK == 4) return table_kernel_mixed_ptr(D, 0, W);
  return nullptr;
}

const void* table_split_kernel_ptr(int D, int PK, int PW, int S) {
  static SplitKernelTab tab = {};
  static bool init = [] {
    split_register_d1(tab);
    split_register_d2(tab);
    split_register_d3(tab);
    split_register_d4_6(tab);
    split_register_d7_10(tab);
    return true;
  }();
  (void)init;
  const int pi = (PW >= 4 && PW <= 32 && PW % 4 == 0) ? PW / 4 - 1 : -1;
  const int si = S == 2 ? 0 : S == 4 ? 1 : S == 8 ? 2 : -1;
  if (D < 1 || D > 10 || (PK != 1 && PK != 4) || pi < 0 || si < 0) return nullptr;
  return tab[D][PK == 4 ? 1 : 0][pi][si];
}

static const PruneKernelTab& prune_kernels() {
  static PruneKernelTab tab = {};
  static bool init = [] {
    prune_register_d1(tab);
    prune_register_d23(tab);
    return true;
  }();
  (void)init;
  return tab;
}

void prune_kernel_ptrs(int D, int WB, int WA, const void** bound, const void** scan) {
  *bound = *scan = nullptr;
  if (D < 1 || D > 3 || WB < 0 || WB > 64 || WA < 0 || WA > 32) return;
  *bound = prune_kernels()[D][WB][WA][0];
  *scan = prune_kernels()[D][WB][WA][1];
}

template <typename IT, bool MULTI, bool SYM>
static const void* wide_pick(int PC) {
  switch (PC) {
    case 1: return (const void*)&wide_kernel<IT, 1, MULTI, SYM>;
    case 2: return (const void*)&wide_kernel<IT, 2, MULTI, SYM>;
    case 4: return (const void*)&wide_kernel<IT, 4, MULTI, SYM>;
    case 8: return (const void*)&wide_kernel<IT, 8, MULTI, SYM>;
    case 16: return (const void*)&wide_kernel<IT, 16, MULTI, SYM>;
    case 32: return (const void*)&wide_kernel<IT, 32, MULTI, SYM>;
    case 64: return (const void*)&wide_kernel<IT, 64, MULTI, SYM>;
    case 128: return (const void*)&wide_kernel<IT, 128, MULTI, SYM>;
    default: return nullptr;
  }
}

// sym: the label-symmetry instance (d >= 3, so multi only)
const void* wide_kernel_ptr(int i64, int PC, int multi, int sym) {
  if (sym && !multi) return nullptr;
  if (i64) {
    if (sym) return wide_pick<long long, true, true>(PC);
    return multi ? wide_pick<long long, true, false>(PC) : wide_pick<long long, false, false>(PC);
  }
  if (sym) return wide_pick<int, true, true>(PC);
  return multi ? wide_pick<int, true, false>(PC) : wide_pick<int, false, false>(PC);
}

}  // namespace ld
