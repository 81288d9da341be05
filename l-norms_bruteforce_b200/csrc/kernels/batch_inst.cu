// Batched persistent kernel instances (lane classes) and their lookup:
//   D = 1: int32 words 8, 16, .., 64 or int8x4 words 4, 8, .., 32
//   D = 2: int32 words 8, 16, .., 64 or int8x4 words 4, 8, .., 32
//   D = 3: int32 words 8, 16, .., 64 or int8x4 words 4, 8, .., 32
// plus column-split instances of the int32 classes of 40 .. 64 words.
#include <utility>

#include "batch_kernel.cuh"
#include "registry.h"

namespace ld {
namespace {

using BatchTab = const void* [4][65][33];

template <int D, int... I>
void fill_b32(BatchTab& t, std::integer_sequence<int, I...>) {
  ((t[D][8 * (I + 1)][0] = (const void*)&batch_table_kernel<D, 8 * (I + 1), 0>), ...);
}
template <int D, int... I>
void fill_b8(BatchTab& t, std::integer_sequence<int, I...>) {
  ((t[D][0][4 * (I + 1)] = (const void*)&batch_table_kernel<D, 0, 4 * (I + 1)>), ...);
}

const BatchTab& batch_kernels() {
  static BatchTab tab = {};
  static bool init = [] {
    fill_b32<1>(tab, std::make_integer_sequence<int, 8>{});
    fill_b32<2>(tab, std::make_integer_sequence<int, 8>{});
    fill_b32<3>(tab, std::make_integer_sequence<int, 8>{});
    fill_b8<1>(tab, std::make_integer_sequence<int, 8>{});
    fill_b8<2>(tab, std::make_integer_sequence<int, 8>{});
    fill_b8<3>(tab, std::make_integer_sequence<int, 8>{});
    return true;
  }();
  (void)init;
  return tab;
}

}  // namespace

const void* batch_kernel_ptr(int D, int WB, int WA) {
  if (D < 1 || D > 3 || WB < 0 || WB > 64 || WA < 0 || WA > 32) return nullptr;
  return batch_kernels()[D][WB][WA];
}

const void* batch_split_kernel_ptr(int D, int WB) {
  // column-split instances: int32 words 40, 48, 56, 64
  static const void* const tab[4][4] = {
      {nullptr, nullptr, nullptr, nullptr},
      {(const void*)&batch_split_kernel<1, 40>, (const void*)&batch_split_kernel<1, 48>,
       (const void*)&batch_split_kernel<1, 56>, (const void*)&batch_split_kernel<1, 64>},
      {(const void*)&batch_split_kernel<2, 40>, (const void*)&batch_split_kernel<2, 48>,
       (const void*)&batch_split_kernel<2, 56>, (const void*)&batch_split_kernel<2, 64>},
      {(const void*)&batch_split_kernel<3, 40>, (const void*)&batch_split_kernel<3, 48>,
       (const void*)&batch_split_kernel<3, 56>, (const void*)&batch_split_kernel<3, 64>}};
  if (D < 1 || D > 3 || !batch_split_class(WB, 0) || WB > 64) return nullptr;
  return tab[D][(WB - 40) / 8];
}

const void* batch_fold_kernel_ptr() { return (const void*)&batch_fold_kernel<0>; }

}  // namespace ld
