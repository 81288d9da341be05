// Pruned-search kernels for D = 2 and D = 3.
#include "prune_inst.cuh"
namespace ld {
void prune_register_d23(PruneKernelTab& t) {
  pinst::fill_wb4<2>(t, std::make_integer_sequence<int, 12>{});
  pinst::fill_wa4<2>(t, std::make_integer_sequence<int, 8>{});
  pinst::fill_wb4<3>(t, std::make_integer_sequence<int, 8>{});
  pinst::fill_wa4<3>(t, std::make_integer_sequence<int, 8>{});
}
}  // namespace ld
