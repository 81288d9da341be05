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

const void* table_kernel_pair_ptr(int WB, int WA, int lin) {
  static TableKernelPairTab tab = {};
  static bool init = [] {
    table_register_pair(tab);
    return true;
  }();
  (void)init;
  if (WB < 0 || WB > 10 || WA < 0 || WA > 16 || WB + WA > 10) return nullptr;
  return tab[lin ? 1 : 0][WB][WA];
}

const void* table_kernel_ptr(int D, int W, int PK) {
  if (PK == 1) return table_kernel_mixed_ptr(D, W, 0);
  if (PK == 4) return table_kernel_mixed_ptr(D, 0, W);
  return nullptr;
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

template <typename IT, bool MULTI>
static const void* wide_pick(int PC) {
  switch (PC) {
    case 1: return (const void*)&wide_kernel<IT, 1, MULTI>;
    case 2: return (const void*)&wide_kernel<IT, 2, MULTI>;
    case 4: return (const void*)&wide_kernel<IT, 4, MULTI>;
    case 8: return (const void*)&wide_kernel<IT, 8, MULTI>;
    case 16: return (const void*)&wide_kernel<IT, 16, MULTI>;
    case 32: return (const void*)&wide_kernel<IT, 32, MULTI>;
    case 64: return (const void*)&wide_kernel<IT, 64, MULTI>;
    case 128: return (const void*)&wide_kernel<IT, 128, MULTI>;
    default: return nullptr;
  }
}

const void* wide_kernel_ptr(int i64, int PC, int multi) {
  if (i64) return multi ? wide_pick<long long, true>(PC) : wide_pick<long long, false>(PC);
  return multi ? wide_pick<int, true>(PC) : wide_pick<int, false>(PC);
}

}  // namespace ld
