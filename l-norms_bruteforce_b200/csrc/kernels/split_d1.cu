// table_split_kernel<D, PK, PW, S> for D = 1: 32-bit lanes with PW = 16, 20,
// .., 32 words per lane and 8-bit lanes with PW = 8, 12, 16, each for S = 2,
// 4, 8 lanes per high index (up to 256 int32 / 512 8-bit columns; the finer
// widths keep the padding of a row to S x PW words small).  Two high
// indices per group (K = 2).
#include "split_inst.cuh"
namespace ld {
namespace {
template <int D, int PK, int PW>
void put_s(SplitKernelTab& t) {
  inst::split_put<D, PK, PW, 2>(t);
  inst::split_put<D, PK, PW, 4>(t);
  inst::split_put<D, PK, PW, 8>(t);
}
}  // namespace
void split_register_d1(SplitKernelTab& t) {
  put_s<1, 1, 16>(t);
  put_s<1, 1, 20>(t);
  put_s<1, 1, 24>(t);
  put_s<1, 1, 28>(t);
  put_s<1, 1, 32>(t);
  put_s<1, 4, 8>(t);
  put_s<1, 4, 12>(t);
  put_s<1, 4, 16>(t);
}
}  // namespace ld
