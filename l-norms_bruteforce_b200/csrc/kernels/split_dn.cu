// table_split_kernel<D, PK, PW, S> for D = 4 .. 10 (register vectors D x PW):
//   D = 4:     32-bit lanes (S, PW) in (2, 16), (4, 16), (8, 16), (8, 32)
//   D = 4..8:  also 32-bit lanes (2, 12), (4, 12), (8, 12)
//   D = 5..8:  32-bit lanes (2, 16), (4, 16), (8, 16)
//   D = 9, 10: 32-bit lanes (2, 8), (4, 8), (8, 8)
//   every D:   8-bit lanes (2, 8), (4, 8), (8, 8)
#include "split_inst.cuh"
namespace ld {
namespace {
template <int D>
void put_d(SplitKernelTab& t) {
  if constexpr (D <= 8) {
    inst::split_put<D, 1, 12, 2>(t);
    inst::split_put<D, 1, 12, 4>(t);
    inst::split_put<D, 1, 12, 8>(t);
    inst::split_put<D, 1, 16, 2>(t);
    inst::split_put<D, 1, 16, 4>(t);
    inst::split_put<D, 1, 16, 8>(t);
  } else {
    inst::split_put<D, 1, 8, 2>(t);
    inst::split_put<D, 1, 8, 4>(t);
    inst::split_put<D, 1, 8, 8>(t);
  }
  if constexpr (D == 4) inst::split_put<D, 1, 32, 8>(t);
  inst::split_put<D, 4, 8, 2>(t);
  inst::split_put<D, 4, 8, 4>(t);
  inst::split_put<D, 4, 8, 8>(t);
}
}  // namespace
void split_register_d4_6(SplitKernelTab& t) { put_d<4>(t); put_d<5>(t); put_d<6>(t); }
void split_register_d7_10(SplitKernelTab& t) { put_d<7>(t); put_d<8>(t); put_d<9>(t); put_d<10>(t); }
}  // namespace ld
