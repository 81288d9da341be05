// Helpers that fill the pruned-search kernel lookup with instances.
#pragma once
#include <utility>

#include "prune_kernel.cuh"
#include "registry.h"

namespace ld {
namespace pinst {

template <int D, int WB, int WA>
void put(PruneKernelTab& t) {
  if constexpr (WB + WA > 0) {
    t[D][WB][WA][0] = (const void*)&walk_bound_kernel<D, WB, WA>;
    t[D][WB][WA][1] = (const void*)&prune_scan_kernel<D, WB, WA>;
  }
}
template <int D, int WB, int... I>
void fill_wa(PruneKernelTab& t, std::integer_sequence<int, I...>) { (put<D, WB, I>(t), ...); }
// WB = 4 (i + 1) for i in I..., WA = 0
template <int D, int... I>
void fill_wb4(PruneKernelTab& t, std::integer_sequence<int, I...>) { (put<D, 4 * (I + 1), 0>(t), ...); }
// WA = 4 (i + 1) for i in I..., WB = 0
template <int D, int... I>
void fill_wa4(PruneKernelTab& t, std::integer_sequence<int, I...>) { (put<D, 0, 4 * (I + 1)>(t), ...); }

}  // namespace pinst
}  // namespace ld
