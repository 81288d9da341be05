// table_kernel instances for D = 1: int32 lanes (PK = 1) for W = 4..64 words,
// int8x4 lanes (PK = 4) for W = 4..32 words.
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
  if (PK == 1) return pick_d1<1>(W, std::make_integer_sequence<int, 16>{});
  if (PK == 4) return pick_d1<4>(W, std::make_integer_sequence<int, 8>{});
  return nullptr;
}

}  // namespace ld
