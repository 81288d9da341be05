// table_kernel instances for D = 1.
#include <utility>

#include "registry.h"
#include "table_kernel.cuh"

namespace ld {

template <int PK, int... Ws>
static const void* pick_d1(int W, std::integer_sequence<int, Ws...>) {
  const void* r = nullptr;
  ((W == (Ws + 1) * 4 ? (r = (const void*)&table_kernel<1, (Ws + 1) * 4, PK>, 0) : 0), ...);
  return r;
}

const void* table_kernel_ptr_d1(int W, int PK) {
  using Seq = std::make_integer_sequence<int, 8>;
  if (PK == 1) return pick_d1<1>(W, Seq{});
  if (PK == 2) return pick_d1<2>(W, Seq{});
  if (PK == 4) return pick_d1<4>(W, Seq{});
  return nullptr;
}

}  // namespace ld
