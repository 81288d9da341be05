// table_kernel<1, WB, 0>: WB = 35..64 int32 words.
#include "table_inst.cuh"
namespace ld {
void table_register_d1_p32b(TableKernelTab& t) {
  inst::fill_wb<1, 0, 35>(t, std::make_integer_sequence<int, 30>{});
}
}  // namespace ld
