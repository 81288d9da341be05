// Declarations shared by the solver's translation units: the kernel choice
// and packing, device resources, plans (solver.cu), the pruned search
// (prune.cu), batches (batch.cu) and resumable solves (resumable.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <mutex>
#include <vector>

#include "../host/ld_internal.h"
#include "../kernels/common.cuh"

#define LD_CUDA(call)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      return ld_fail(e_ == cudaErrorNoDevice || e_ == cudaErrorInsufficientDriver       \
                         ? LD_ERR_NODEV : LD_ERR_CUDA,                                  \
                     "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    }                                                                                   \
  } while (0)

namespace ldsolve {

// Exact bounds on every quantity a kernel forms.
struct Bounds {
  long long colbound;   // max over columns of sum_i |A_il|: any partial column sum
  long long total;      // sum of |A_il|: any labeling's value
  long long K;          // LM: sum_i |A_i0| (column-0 shift)
  bool overflow;        // a bound itself exceeds int64
};

Bounds compute_bounds(const int64_t* a, int R, int C, int marginal);

struct Choice {
  int kind = LD_KERNEL_WIDE;
  int D = 0, WB = 0, WA = 0, WT = 0, k = 0;   // table: int32 words, int8x4 words, padded, low rows
  std::vector<int> order;                     // table: column of each lane (wide first)
  int PC = 0, multi = 0, i64 = 0;             // wide
  int lane_bits = 0;
  int lin = 0;                                // table: LM column 0 linear in word 0
  int pair = 0;                               // table: two high indices per thread
  int S = 0, PW = 0, PK = 0;                  // column-split table kernel: lanes per high
                                              // index, words per lane, columns per word
};

inline int round4(int x) { return (x + 3) & ~3; }

inline unsigned long long ipow(unsigned long long b, int e) {
  unsigned long long r = 1;
  for (int i = 0; i < e; ++i) r *= b;
  return r;
}

bool table_config(const int64_t* a, int R, int C, int d, int marginal, int k, int force_bits, Choice* ch);
int split_bank_pad(int S, int NW, int span);
ld_status choose_kernel(const int64_t* a, int R, int C, int d, int marginal, const Bounds& b,
                        const ld_options& o, int sms, Choice* ch);
void pack_row(const int64_t* row, const Choice& ch, uint32_t* out);

struct DeviceInfo {
  int sms = 148;
  int max_threads = 1024;
  bool ok = false;
};

ld_status device_info(int dev, DeviceInfo* out);

// Device resources: one device arena, a pinned staging buffer, a stream and
// three events.  A plan owns its own; ld_solve_reduced borrows a per-device
// workspace (g_ws), the pruned search another (g_pws).
struct Resources {
  int device = -1;
  void* dmem = nullptr;
  size_t dcap = 0;
  void* hstage = nullptr;
  size_t hcap = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
};

void resources_release(Resources* r);
ld_status resources_acquire(Resources* r, int device, cudaStream_t user_stream, size_t dbytes, size_t hbytes);
extern std::mutex g_ws_mu[64];
extern Resources g_ws[64];
extern std::mutex g_pws_mu[64];
extern Resources g_pws[64];

// a plan's device image: reduction header, then totals, initial H, table
// bias and packed rows
constexpr size_t kOffCounter = 0, kOffGvalue = 8, kOffResult = 16, kOffWork = 32;
constexpr size_t kOffTot = 256, kOffH0 = 512, kOffTb = 768, kOffA = 1024;

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

void split_range(unsigned long long n, int idx, int count, unsigned long long* lo, unsigned long long* hi);

}  // namespace ldsolve

struct ld_plan {
  int device = 0;
  int R = 0, C = 0, d = 0, marginal = 0;
  ldsolve::Choice ch;
  ldsolve::Bounds bounds{};
  int k = 0, B = 1, fw = 0;                       // table geometry
  // walks: the table kernel's blocks of high indices, or (wide kernel with
  // label symmetry) runs of walk_len consecutive indices
  unsigned long long walk_len = 1, walks = 1, walk_begin = 0, walk_end = 1;
  int sym_digits = 0;                             // label symmetry: walk-number digits
  size_t sym_off = 0;                             // completion counts in the device image
  unsigned long long rank_begin = 0, rank_end = 0;  // passing walks of the shard, by rank
  unsigned long long walks_run = 1;               // walks of [walk_begin, walk_end) that pass
  unsigned long long n_begin = 0, n_end = 0;      // wide geometry
  unsigned long long total = 0;
  int blocks = 1, tpb = 128;
  size_t smem = 0;
  long long value_offset = 0;
  ldsolve::Resources own;
  ldsolve::Resources* res = nullptr;
  size_t upload_bytes = 0;
  // table kernels: image offsets of the totals, initial H, table bias and rows
  size_t off_tot = 0, off_h0 = 0, off_tb = 0, off_A = 0;
  int Bp = 0, span = 0;                           // column split: table entries, words per slice region
  int pack16 = 0;                                 // table kernel: packed 16-bit maxima
  bool uploaded = false;       // the upload belongs to the next fetched launch
  ld::Reduce red{};
  const void* kfn = nullptr;
  bool launched = false;
};

namespace ldsolve {

void plan_free(ld_plan* p);
// geometry, kernel choice and the upload image; `shared` selects a
// per-device workspace instead of the plan's own resources
ld_status plan_build(const int64_t* a, int R, int C, int d, int marginal, const ld_options* opt,
                     Resources* shared, ld_plan** out);
ld_status plan_enqueue(ld_plan* p);
unsigned long long plan_evaluated(const ld_plan* p);
ld_status plan_fetch(ld_plan* p, ld_result* res, int32_t* strategy);

}  // namespace ldsolve
