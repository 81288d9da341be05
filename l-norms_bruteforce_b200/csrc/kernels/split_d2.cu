// table_split_kernel<D, PK, PW, S> for D = 2: 32-bit lanes with
// (S, PW) in (2, 32), (4, 32), (8, 16), (8, 32) (up to 256 columns), 8-bit
// lanes with (2, 16), (4, 16), (8, 16) (up to 512 columns).
#include "split_inst.cuh"
namespace ld {
namespace {
template <int D>
void put_d(SplitKernelTab& t) {
  inst::split_put<D, 1, 32, 2>(t);
  inst::split_put<D, 1, 32, 4>(t);
  inst::split_put<D, 1, 16, 8>(t);
  inst::split_put<D, 1, 32, 8>(t);
  inst::split_put<D, 4, 16, 2>(t);
  inst::split_put<D, 4, 16, 4>(t);
  inst::split_put<D, 4, 16, 8>(t);
}
}  // namespace
void split_register_d2(SplitKernelTab& t) { put_d<2>(t); }
}  // namespace ld
