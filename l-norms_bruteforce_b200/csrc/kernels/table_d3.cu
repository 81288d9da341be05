// table_kernel<3, WB, 0> for WB = 1..64 and table_kernel<3, 0, WA> for WA = 1..32.
#include "table_inst.cuh"
namespace ld {
void table_register_d3(TableKernelTab& t) {
  inst::fill_wb<3, 0, 1>(t, std::make_integer_sequence<int, 64>{});
  inst::fill_wa<3, 0, 1>(t, std::make_integer_sequence<int, 32>{});
}
}  // namespace ld
