// table_kernel<1, WB, WA, LIN, PAIR = true>: L_1 / LM with WB + WA <= 10 words
// (two high indices per thread against each table entry read).
#include "table_inst.cuh"
namespace ld {
namespace {
template <bool LIN, int WB, int WA>
constexpr const void* pair_kp() {
  if constexpr (WB + WA == 0 || WB + WA > 10 || (LIN && WB == 0)) return nullptr;
  else return (const void*)&table_kernel<1, WB, WA, LIN, true>;
}
template <bool LIN, int WB, int... I>
void fill_pair(TableKernelPairTab& t, std::integer_sequence<int, I...>) {
  ((t[LIN ? 1 : 0][WB][I] = pair_kp<LIN, WB, I>()), ...);
}
}  // namespace
void table_register_pair(TableKernelPairTab& t) {
  using Seq = std::make_integer_sequence<int, 11>;
  fill_pair<false, 0>(t, Seq{});
  fill_pair<false, 1>(t, Seq{});
  fill_pair<false, 2>(t, Seq{});
  fill_pair<false, 3>(t, Seq{});
  fill_pair<false, 4>(t, Seq{});
  fill_pair<true, 1>(t, Seq{});
  fill_pair<true, 2>(t, Seq{});
  t[0][5][0] = pair_kp<false, 5, 0>();
  t[0][6][0] = pair_kp<false, 6, 0>();
  t[0][7][0] = pair_kp<false, 7, 0>();
  t[0][8][0] = pair_kp<false, 8, 0>();
  t[0][9][0] = pair_kp<false, 9, 0>();
  t[0][10][0] = pair_kp<false, 10, 0>();
}
}  // namespace ld
