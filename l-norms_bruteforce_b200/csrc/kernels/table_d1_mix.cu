// table_kernel<1, WB, WA>: WB = 0..4 int32 words with WA = 0..16 int8x4 words.
#include "table_inst.cuh"
namespace ld {
void table_register_d1_mix(TableKernelTab& t) {
  using Seq = std::make_integer_sequence<int, 17>;
  inst::fill_wa<1, 0, 0>(t, Seq{});
  inst::fill_wa<1, 1, 0>(t, Seq{});
  inst::fill_wa<1, 2, 0>(t, Seq{});
  inst::fill_wa<1, 3, 0>(t, Seq{});
  inst::fill_wa<1, 4, 0>(t, Seq{});
}
}  // namespace ld
