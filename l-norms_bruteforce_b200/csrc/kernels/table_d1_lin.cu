// table_kernel<1, WB, WA, LIN = true> for LM with the marginal column in
// a 32-bit word of its own: WB = 1..2 int32 words with WA = 0..16 int8x4 words.
#include "table_inst.cuh"
namespace ld {
namespace {
template <int WB, int... I>
void fill_lin(TableKernelLinTab& t, std::integer_sequence<int, I...>) {
  ((t[WB][I] = (const void*)&table_kernel<1, WB, I, true>), ...);
}
}  // namespace
void table_register_d1_lin(TableKernelLinTab& t) {
  using Seq = std::make_integer_sequence<int, 17>;
  fill_lin<1>(t, Seq{});
  fill_lin<2>(t, Seq{});
}
}  // namespace ld
