// table_kernel<D, WB, WA, false, PAIR = true> for D = 2, 3: two high indices
// per thread against each table entry read, with WB in 1..8 (WA = 0) or WA
// in 1..8 (WB = 0) words per message vector.
#include "table_inst.cuh"
namespace ld {
namespace {
template <int D, int WB, int WA>
constexpr const void* pair23_kp() {
  if constexpr (WB + WA == 0) return nullptr;
  else return (const void*)&table_kernel<D, WB, WA, false, true>;
}
template <int D, int... I>
void fill_pair23(TableKernelPair23Tab& t, std::integer_sequence<int, I...>) {
  ((t[D - 2][I][0] = pair23_kp<D, I, 0>()), ...);
  ((t[D - 2][0][I] = pair23_kp<D, 0, I>()), ...);
}
}  // namespace
void table_register_pair23(TableKernelPair23Tab& t) {
  fill_pair23<2>(t, std::make_integer_sequence<int, 9>{});
  fill_pair23<3>(t, std::make_integer_sequence<int, 9>{});
}
}  // namespace ld
