// wide_kernel instances and the kernel registry.
#include "registry.h"
#include "wide_kernel.cuh"

namespace ld {

const void* table_kernel_ptr_d1(int W, int PK);
const void* table_kernel_ptr_d2(int W, int PK);
const void* table_kernel_ptr_d3(int W, int PK);

const void* table_kernel_ptr(int D, int W, int PK) {
  if (D == 1) return table_kernel_ptr_d1(W, PK);
  if (D == 2) return table_kernel_ptr_d2(W, PK);
  if (D == 3) return table_kernel_ptr_d3(W, PK);
  return nullptr;
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
