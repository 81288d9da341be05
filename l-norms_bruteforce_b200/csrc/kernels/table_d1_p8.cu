// table_kernel<1, 0, WA>: WA = 17..32 int8x4 words.
#include "table_inst.cuh"
namespace ld {
void table_register_d1_p8(TableKernelTab& t) {
  inst::fill_wa<1, 0, 17>(t, std::make_integer_sequence<int, 16>{});
}
}  // namespace ld
