// Helpers that fill the column-split kernel lookup with instances.
#pragma once
#include "registry.h"
#include "split_kernel.cuh"

namespace ld {
namespace inst {

constexpr int split_pw_index(int PW) { return PW / 4 - 1; }   // PW = 4, 8, .., 32
constexpr int split_s_index(int S) { return S == 2 ? 0 : S == 4 ? 1 : 2; }

// K: high indices per group (2 for d <= 2, whose one register vector per
// high index leaves room for two)
template <int D, int PK, int PW, int S, int K = (D <= 2 ? 2 : 1)>
void split_put(SplitKernelTab& t) {
  t[D][PK == 4 ? 1 : 0][split_pw_index(PW)][split_s_index(S)] = (const void*)&table_split_kernel<D, PK, PW, S, K>;
}

}  // namespace inst
}  // namespace ld
