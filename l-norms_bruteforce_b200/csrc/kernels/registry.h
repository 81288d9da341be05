// Kernel instances, compiled in separate translation units.
#pragma once

namespace ld {
// table_kernel<D, W, PK> for D in {1,2,3}, W in {4,8,...,32}, PK in {1,2,4};
// nullptr when not instantiated.
const void* table_kernel_ptr(int D, int W, int PK);
// wide_kernel<IT, PC, MULTI>, PC in {1,2,4,...,128}
const void* wide_kernel_ptr(int i64, int PC, int multi);
}  // namespace ld

#define LD_WIDE_MAXD 10
