// ld_solve_reduced_noalloc: the exact solve without any device allocation.
//
// Who needs it: callers that are not allowed to allocate GPU memory at the
// time they solve.  cudaMalloc and cudaFree can synchronize the whole device
// and can fail once another framework in the process (a training loop, an
// inference server) has reserved nearly all of the GPU's memory for its own
// pool; code that runs inside such a process, or inside a latency-bound loop
// that must not stall other streams, cannot call them.  ld_solve_reduced
// allocates on its first call per device and ld_plan_create on every call;
// this entry point never does.
//
// How: all device-side working memory -- the packed matrix image the table
// kernel reads, its per-block result slots, the completion counter, the
// running maximum and the final result -- lives in one file-scope
// __device__ array, g_noalloc_scratch, of kNoallocScratchBytes (64 KiB).
// Every GPU that loads this library reserves it until the process exits.
// The caller passes the matrix and receives the result in host memory, as
// with ld_solve_reduced.
//
// Set-up: host code cannot use the array's name as a device address (in
// host code it names a host-side stand-in).  The first call on each device
// makes that device current and looks the address up with
// cudaGetSymbolAddress, once; make the first call on a device before any
// stream capture on it.
//
// Stream: the work goes to the caller's stream; NULL means the legacy
// default stream, which waits for (and holds up) every blocking stream of
// the device, so a caller that must not stall other work passes a stream
// created with cudaStreamNonBlocking.  Every call waits for its stream to
// finish before it returns the result.
//
// Sharing: every call uses the same array and it keeps the previous call's
// contents.  Each call rewrites the image and the counter / running-maximum
// words that must start at 0 / INT64_MIN.  Calls from host threads of this
// process are serialised by a lock held until the call's stream has
// finished; work issued to the same device by other means while a call runs
// does not touch the array, but two calls whose GPU work overlapped (for
// example from code that bypasses this function's lock) would race on it.
//
// Limit: the table kernel only (d <= 3; up to 64 columns in 32-bit lanes,
// 128 in 8-bit lanes; at most 63 rows), so that the image (at most 16.5 KiB),
// the label-symmetry counts of d = 3 (at most 2.5 KiB) and one 16-byte slot per
// block fit in the 64 KiB array.  Anything larger is rejected with
// LD_ERR_LIMIT before any device work.  The work is ld_solve_reduced's: at
// d = 3 the walks that cannot hold the smallest index of a class of
// label-permuted labelings are skipped there too.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <mutex>

#include "smem_limit.h"
#include "../host/ld_internal.h"
#include "../kernels/common.cuh"
#include "../kernels/registry.h"
#include "../kernels/table_kernel.cuh"
#include "device_guard.h"

namespace {

constexpr size_t kNoallocScratchBytes = 64 * 1024;

// The scratch array.  Device code could name it directly; host code only
// uses the address returned by cudaGetSymbolAddress.
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

// image layout: the allocating path's upload image without its table-bias
// block, so the rows start at 768.  No bias is needed: for LM the whole shift
// K = sum |A_i0| goes into the initial high sums (h0[0] += K) and is
// subtracted from the value; the table then holds the low rows' signed part
// alone, which stays within 8 bits whenever 8-bit lanes are chosen
// (2K <= 127).  The d = 3 label-symmetry counts follow the rows, 256-byte
// aligned.
constexpr size_t kCounter = 0, kGvalue = 8, kResult = 16;
constexpr size_t kTot = 256, kH0 = 512, kA = 768;
constexpr size_t kMaxRows = kA + 63 * 64 * 4;     // 63 rows x 64 words
constexpr size_t kMaxSym = 4096;                  // d = 3: 8 (P + 1) counts of 8 bytes, P <= 39
constexpr size_t kMaxImage = ((kMaxRows + 255) & ~(size_t)255) + kMaxSym;

std::mutex g_mu[64];
void* g_scratch[64];          // device address of the array, per device
int g_sms[64];

size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

uint32_t pack(const int64_t* v, int n, int pk) {
  const int bits = 32 / pk;
  const uint32_t mask = bits == 32 ? 0xffffffffu : ((1u << bits) - 1u);
  uint32_t w = 0;
  for (int q = 0; q < pk && q < n; ++q) w |= ((uint32_t)(int32_t)v[q] & mask) << (q * bits);
  return w;
}

void pack_row(const int64_t* row, int C, int W, int pk, uint32_t* out) {
  for (int w = 0; w < W; ++w) {
    const int c0 = w * pk;
    out[w] = c0 < C ? pack(row + c0, std::min(pk, C - c0), pk) : 0u;
  }
}

unsigned long long ipow(unsigned long long b, int e) {
  unsigned long long r = 1;
  for (int i = 0; i < e; ++i) r *= b;
  return r;
}

}  // namespace

extern "C" ld_status ld_solve_reduced_noalloc(const int64_t* a, int32_t R, int32_t C, int32_t d,
                                              int32_t marginal, int32_t device, void* stream,
                                              ld_result* res, int32_t* strategy) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
  if (!a || !res || R < 1 || C < 1) return ld_fail(LD_ERR_ARG, "bad arguments");
  if (d < 1 || d > 3) return ld_fail(LD_ERR_LIMIT, "no-allocation solve takes d = 1, 2 or 3 (got %d)", d);
  if (marginal && d != 1) return ld_fail(LD_ERR_ARG, "marginals need d == 1");
  if (R > 63) return ld_fail(LD_ERR_LIMIT, "no-allocation solve takes at most 63 rows (got %d)", R);
  if (device < 0 || device >= 64) return ld_fail(LD_ERR_ARG, "device %d out of range", device);
  if (ld_labelings(R, d) >= (1ull << 63)) return ld_fail(LD_ERR_LIMIT, "too many labelings");

  // exact bounds -> lane width (8-bit lanes when every partial column sum
  // fits, else 32-bit)
  long long colbound = 0, total = 0, K = 0;
  for (int l = 0; l < C; ++l) {
    long long s = 0;
    for (int i = 0; i < R; ++i) {
      const long long v = a[(size_t)i * C + l];
      const long long av = v < 0 ? -v : v;
      if (av > (long long)INT32_MAX) return ld_fail(LD_ERR_LIMIT, "entries exceed the 32-bit range");
      s += av;
    }
    colbound = std::max(colbound, s);
    total += s;
    if (l == 0 && marginal) K = s;
  }
  const long long maxabs = std::max(colbound, marginal ? 2 * K : 0LL);
  if (total + K > (long long)INT32_MAX)
    return ld_fail(LD_ERR_LIMIT, "no-allocation solve needs column sums within 32 bits");
  int PK = 0, W = 0;
  if (maxabs <= 127 && (C + 3) / 4 <= 32) { PK = 4; W = (((C + 3) / 4) + 3) & ~3; }
  else {
    PK = 1; W = (C + 3) & ~3;
    if (W > 64) return ld_fail(LD_ERR_LIMIT, "no-allocation solve takes at most 64 columns (got %d)", C);
  }
  const void* kfn = ld::table_kernel_ptr(d, W, PK);
  if (!kfn) return ld_fail(LD_ERR_LIMIT, "no table kernel for d=%d and %d columns", d, C);

  std::lock_guard<std::mutex> lk(g_mu[device]);
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return ld_fail(LD_ERR_NODEV, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
  if (!g_scratch[device]) {                       // once per device
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return ld_fail(LD_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return ld_fail(LD_ERR_CUDA, "device attribute: %s", cudaGetErrorString(e));
    g_sms[device] = sms;
    g_scratch[device] = p;
  }
  char* scratch = (char*)g_scratch[device];
  cudaStream_t st = (cudaStream_t)stream;

  // geometry (same rules as the allocating path)
  const int base = d <= 2 ? 2 : d, F = R - 1, NW = d * W;
  const int maxB = std::min(1024, 8192 / NW);
  int k = 0;
  while (k < F && ipow(base, k + 1) <= (unsigned long long)maxB) ++k;
  const int B = (int)ipow(base, k);
  const size_t smem = (size_t)ld::table_smem_words(d, W, R, B) * sizeof(uint32_t);
  e = ld_raise_smem_limit(kfn, smem);
  if (e != cudaSuccess) return ld_fail(LD_ERR_CUDA, "shared memory attribute: %s", cudaGetErrorString(e));
  int bps = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kfn, ld::kTableThreads, smem);
  if (e != cudaSuccess || bps < 1) return ld_fail(LD_ERR_CUDA, "occupancy query failed");
  const unsigned long long full = (unsigned long long)g_sms[device] * bps * ld::kTableThreads;
  const int nh = F - k;
  // d = 3: only the walks that can hold a class minimum run (label
  // symmetry), handed out by rank; the walk length follows the allocating
  // path's rule (walks that run >= 16 per thread of a full grid for d <= 2,
  // >= 4 for d = 3)
  const bool sym = d >= 3;
  auto walks_run = [&](int f) -> unsigned long long {
    uint64_t c = ipow(base, nh - f);
    if (sym && nh - f > 0 && ld_symmetry_walks(d, nh - f, 0, c, &c) != LD_OK) c = ipow(base, nh - f);
    return (unsigned long long)c;
  };
  const unsigned long long per_thread = d >= 3 ? 4ull : 16ull;
  int fw = 0;
  while (fw < nh && walks_run(fw + 1) >= per_thread * full) ++fw;
  const unsigned long long walk_len = ipow(base, fw), walks = ipow(base, nh - fw);
  const int P = sym ? nh - fw : 0;
  const unsigned long long run = walks_run(fw);
  const size_t rows_end = kA + (size_t)R * W * 4;
  const size_t sym_off = up256(rows_end);
  const size_t sym_bytes = P > 0 ? ld_sym_table_len(d, P) * sizeof(uint64_t) : 0;
  const size_t image = P > 0 ? sym_off + sym_bytes : rows_end;
  if (rows_end > kMaxRows || sym_bytes > kMaxSym || image > kMaxImage)
    return ld_fail(LD_ERR_LIMIT, "matrix image exceeds the scratch array");
  const size_t off_slots = up256(image);
  const unsigned long long max_blocks = (kNoallocScratchBytes - off_slots) / sizeof(ld::Slot);
  unsigned long long blocks = std::min<unsigned long long>((unsigned long long)g_sms[device] * bps,
                                                           std::max(1ull, (run + ld::kTableThreads - 1) / ld::kTableThreads));
  blocks = std::min(blocks, max_blocks);
  if (blocks < 1) return ld_fail(LD_ERR_LIMIT, "matrix image exceeds the scratch array");

  // upload image, built in a host stack buffer: header (counter 0, maximum
  // INT64_MIN), totals, initial H, packed rows
  alignas(16) unsigned char img[kMaxImage];
  memset(img, 0, image);
  const long long gmin = LLONG_MIN;
  memcpy(img + kGvalue, &gmin, sizeof gmin);
  int64_t tot[128], h0[128];
  for (int l = 0; l < C; ++l) { tot[l] = 0; h0[l] = 0; }
  for (int i = 0; i < R; ++i)
    for (int l = 0; l < C; ++l) tot[l] += a[(size_t)i * C + l];
  long long offset = 0;
  if (d == 1) {
    for (int l = 0; l < C; ++l) h0[l] = a[(size_t)(R - 1) * C + l];
    if (marginal) { h0[0] += K; offset = K; }
  }
  pack_row(tot, C, W, PK, (uint32_t*)(img + kTot));
  pack_row(h0, C, W, PK, (uint32_t*)(img + kH0));
  for (int i = 0; i < R; ++i) pack_row(a + (size_t)i * C, C, W, PK, (uint32_t*)(img + kA) + (size_t)i * W);
  if (P > 0) {
    const ld_status sst = ld_sym_table(d, P, (uint64_t*)(img + sym_off));
    if (sst != LD_OK) return sst;
  }
  e = cudaMemcpyAsync(scratch, img, image, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return ld_fail(LD_ERR_CUDA, "upload: %s", cudaGetErrorString(e));

  ld::TableArgs args;
  args.A = (const uint32_t*)(scratch + kA);
  args.tot = (const uint32_t*)(scratch + kTot);
  args.hinit = (const uint32_t*)(scratch + kH0);
  args.tbias = nullptr;
  args.R = R; args.k = k; args.B = B; args.fw = fw;
  args.walk_len = walk_len; args.walk_begin = 0; args.walk_end = walks;
  args.sym_digits = P;
  args.sym_table = (const unsigned long long*)(scratch + sym_off);
  args.rank_begin = 0;
  args.rank_end = P > 0 ? run : 0;
  args.value_offset = offset;
  args.pack16 = 0;
  args.red.counter = (unsigned int*)(scratch + kCounter);
  args.red.gvalue = (long long*)(scratch + kGvalue);
  args.red.result = (ld::Slot*)(scratch + kResult);
  args.red.slots = (ld::Slot*)(scratch + off_slots);
  args.red.work = nullptr;   // walks split statically
  void* params[] = {&args};
  e = cudaLaunchKernel(kfn, dim3((unsigned)blocks), dim3(ld::kTableThreads), params, smem, st);
  if (e != cudaSuccess) return ld_fail(LD_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
  ld::Slot out;
  e = cudaMemcpyAsync(&out, scratch + kResult, sizeof out, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return ld_fail(LD_ERR_CUDA, "result: %s", cudaGetErrorString(e));
  memset(res, 0, sizeof *res);
  res->value = out.value;
  res->gray_index = out.index;
  res->labelings = walks * walk_len * (unsigned long long)B;
  res->evaluated = run * walk_len * (unsigned long long)B;
  res->kernel_kind = LD_KERNEL_TABLE;
  res->lane_bits = 32 / PK;
  res->h2d_bytes = image;
  res->d2h_bytes = sizeof out;
  if (strategy) ld_gray_labels(out.index, R, d, strategy);
  return LD_OK;
}
