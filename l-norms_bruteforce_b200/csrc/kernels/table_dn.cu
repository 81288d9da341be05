// table_kernel<D, WB, WA> for D = 4..10 (L_4 .. L_10): WA = 1..8 int8x4
// words, or WB = 4, 8, 12, 16 int32 words (columns padded to a multiple of 4).
#include "table_inst.cuh"
namespace ld {
namespace {
template <int D>
void fill_dn(TableKernelTab& t) {
  inst::fill_wa<D, 0, 1>(t, std::make_integer_sequence<int, 8>{});
  t[D][4][0] = inst::kp<D, 4, 0>();
  t[D][8][0] = inst::kp<D, 8, 0>();
  t[D][12][0] = inst::kp<D, 12, 0>();
  t[D][16][0] = inst::kp<D, 16, 0>();
}
}  // namespace
void table_register_dn(TableKernelTab& t) {
  fill_dn<4>(t);
  fill_dn<5>(t);
  fill_dn<6>(t);
  fill_dn<7>(t);
  fill_dn<8>(t);
  fill_dn<9>(t);
  fill_dn<10>(t);
}
}  // namespace ld
