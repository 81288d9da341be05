// table_kernel<1, WB, 0>: WB = 5..34 int32 words.
#include "table_inst.cuh"
namespace ld {
void table_register_d1_p32a(TableKernelTab& t) {
  inst::fill_wb<1, 0, 5>(t, std::make_integer_sequence<int, 30>{});
}
}  // namespace ld
