// Helpers that fill the table-kernel lookup with instances.
#pragma once
#include <utility>

#include "registry.h"
#include "table_kernel.cuh"

namespace ld {
namespace inst {

template <int D, int WB, int WA>
constexpr const void* kp() {
  if constexpr (WB + WA == 0) return nullptr;
  else return (const void*)&table_kernel<D, WB, WA>;
}
// WA = WA0 + i for i in I..., fixed WB
template <int D, int WB, int WA0, int... I>
void fill_wa(TableKernelTab& t, std::integer_sequence<int, I...>) {
  ((t[D][WB][WA0 + I] = kp<D, WB, WA0 + I>()), ...);
}
// WB = WB0 + i for i in I..., fixed WA
template <int D, int WA, int WB0, int... I>
void fill_wb(TableKernelTab& t, std::integer_sequence<int, I...>) {
  ((t[D][WB0 + I][WA] = kp<D, WB0 + I, WA>()), ...);
}

}  // namespace inst
}  // namespace ld
