// table_kernel<2, WB, 0> for WB = 1..64 and table_kernel<2, 0, WA> for WA = 1..32.
#include "table_inst.cuh"
namespace ld {
void table_register_d2(TableKernelTab& t) {
  inst::fill_wb<2, 0, 1>(t, std::make_integer_sequence<int, 64>{});
  inst::fill_wa<2, 0, 1>(t, std::make_integer_sequence<int, 32>{});
}
}  // namespace ld
