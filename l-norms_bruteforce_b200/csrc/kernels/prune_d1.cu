// Pruned-search kernels for D = 1.
#include "prune_inst.cuh"
namespace ld {
void prune_register_d1(PruneKernelTab& t) {
  using S17 = std::make_integer_sequence<int, 17>;
  pinst::fill_wa<1, 0>(t, S17{});
  pinst::fill_wa<1, 1>(t, S17{});
  pinst::fill_wa<1, 2>(t, S17{});
  pinst::fill_wb4<1>(t, std::make_integer_sequence<int, 16>{});
}
}  // namespace ld
