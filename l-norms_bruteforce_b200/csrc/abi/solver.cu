// Solver orchestration: kernel choice from exact bounds, packing, launch
// geometry, plans, and the calc_Lnorm replacement ld_solve_reduced.
//
// The reference launches one kernel with a user-given grid, has every
// thread write its best value and full strategy to global memory, copies
// copyNum*(R-1) ints back and takes the argmax on the host (L_CUDA.cu:281-359).
// Here the grid is sized from the SM count and the kernel's occupancy, the
// reduction to (value, smallest Gray index) happens on the device, and the
// host reads 16 bytes; the strategy is rebuilt from the Gray index.
#include <cuda_runtime.h>

#include <algorithm>
#include <cinttypes>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "../host/ld_internal.h"
#include "../kernels/common.cuh"
#include "../kernels/registry.h"
#include "../kernels/table_kernel.cuh"
#include "../kernels/wide_kernel.cuh"

namespace {

#define LD_CUDA(call)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      return ld_fail(e_ == cudaErrorNoDevice || e_ == cudaErrorInsufficientDriver       \
                         ? LD_ERR_NODEV : LD_ERR_CUDA,                                  \
                     "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    }                                                                                   \
  } while (0)

// Exact bounds on every quantity a kernel forms.
struct Bounds {
  long long colbound;   // max over columns of sum_i |A_il|: any partial column sum
  long long total;      // sum of |A_il|: any labeling's value
  long long K;          // LM: sum_i |A_i0| (column-0 shift)
  bool overflow;        // a bound itself exceeds int64
};

Bounds compute_bounds(const int64_t* a, int R, int C, int marginal) {
  Bounds b{0, 0, 0, false};
  for (int l = 0; l < C; ++l) {
    unsigned __int128 s = 0;
    for (int i = 0; i < R; ++i) {
      int64_t v = a[(size_t)i * C + l];
      s += (unsigned __int128)(v < 0 ? -(__int128)v : (__int128)v);
    }
    if (s > (unsigned __int128)LLONG_MAX / 4) { b.overflow = true; s = LLONG_MAX / 4; }
    b.colbound = std::max<long long>(b.colbound, (long long)s);
    if (l == 0 && marginal) b.K = (long long)s;
    unsigned __int128 t = (unsigned __int128)b.total + s;
    if (t > (unsigned __int128)LLONG_MAX / 4) { b.overflow = true; t = LLONG_MAX / 4; }
    b.total = (long long)t;
  }
  return b;
}

struct Choice {
  int kind = LD_KERNEL_WIDE;
  int D = 0, W = 0, PK = 0;          // table
  int PC = 0, multi = 0, i64 = 0;    // wide
  int lane_bits = 0;
};

int round4(int x) { return (x + 3) & ~3; }

ld_status choose_kernel(int R, int C, int d, int marginal, const Bounds& b, const ld_options& o,
                        Choice* ch) {
  if (b.overflow) return ld_fail(LD_ERR_LIMIT, "matrix entries too large: column sums exceed 2^61");
  const long long maxabs = std::max(b.colbound, marginal ? 2 * b.K : 0LL);
  const long long vmax = b.total + (marginal ? b.K : 0LL);
  const bool fits32 = vmax <= (long long)INT32_MAX && maxabs <= (long long)INT32_MAX;
  if (o.kernel != LD_KERNEL_WIDE && d <= 3 && o.lane_bits != 64) {
    const int cand[2] = {4, 1};
    for (int pk : cand) {
      const int bits = 32 / pk;
      if (o.lane_bits && o.lane_bits != bits) continue;
      const long long lim = pk == 4 ? 127 : (long long)INT32_MAX;
      if (maxabs > lim || !fits32) continue;
      const int W = round4((C + pk - 1) / pk);
      const int wmax = pk == 4 ? 32 : (d == 1 ? 64 : d == 2 ? 48 : 32);
      if (W > wmax) continue;
      ch->kind = LD_KERNEL_TABLE; ch->D = d; ch->W = W; ch->PK = pk; ch->lane_bits = bits;
      return LD_OK;
    }
    if (o.kernel == LD_KERNEL_TABLE)
      return ld_fail(LD_ERR_ARG, "the table kernel cannot take this matrix (d=%d, %d columns)", d, C);
  }
  ch->kind = LD_KERNEL_WIDE;
  ch->i64 = (!fits32 || o.lane_bits == 64) ? 1 : 0;
  ch->lane_bits = ch->i64 ? 64 : 32;
  if (o.lane_bits == 8)
    return ld_fail(LD_ERR_ARG, "8-bit lanes need the table kernel");
  if (o.lane_bits && o.lane_bits != 32 && o.lane_bits != 64)
    return ld_fail(LD_ERR_ARG, "lane width %d is not 8, 32 or 64", o.lane_bits);
  int pc = 1;
  while (pc * 32 < C) pc *= 2;
  ch->PC = pc;
  ch->multi = d >= 2;
  return LD_OK;
}

uint32_t pack_word(const int64_t* v, int n, int pk) {
  uint32_t w = 0;
  const int bits = 32 / pk;
  const uint32_t mask = bits == 32 ? 0xffffffffu : ((1u << bits) - 1u);
  for (int q = 0; q < pk && q < n; ++q) w |= ((uint32_t)(int32_t)v[q] & mask) << (q * bits);
  return w;
}

void pack_row(const int64_t* row, int C, int W, int pk, uint32_t* out) {
  for (int w = 0; w < W; ++w) {
    const int c0 = w * pk;
    out[w] = c0 < C ? pack_word(row + c0, std::min(pk, C - c0), pk) : 0u;
  }
}

unsigned long long ipow(unsigned long long b, int e) {
  unsigned long long r = 1;
  for (int i = 0; i < e; ++i) r *= b;
  return r;
}

struct DeviceInfo {
  int sms = 148;
  int max_threads = 1024;
  bool ok = false;
};

std::mutex g_dev_mu;
DeviceInfo g_dev[64];

ld_status device_info(int dev, DeviceInfo* out) {
  std::lock_guard<std::mutex> lk(g_dev_mu);
  if (dev < 0 || dev >= 64) return ld_fail(LD_ERR_ARG, "device %d out of range", dev);
  if (!g_dev[dev].ok) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
      return ld_fail(LD_ERR_NODEV, "no CUDA device: %s", e == cudaSuccess ? "count is 0" : cudaGetErrorString(e));
    if (dev >= n) return ld_fail(LD_ERR_NODEV, "device %d not present (%d devices)", dev, n);
    cudaDeviceProp p;
    LD_CUDA(cudaGetDeviceProperties(&p, dev));
    g_dev[dev].sms = p.multiProcessorCount;
    g_dev[dev].max_threads = p.maxThreadsPerBlock;
    g_dev[dev].ok = true;
  }
  *out = g_dev[dev];
  return LD_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Device resources: one device arena, a pinned staging buffer, a stream and
// two events.  A plan owns its own; ld_solve_reduced borrows a per-device
// workspace so repeated calls allocate nothing after the first.
namespace {

struct Resources {
  int device = -1;
  void* dmem = nullptr;
  size_t dcap = 0;
  void* hstage = nullptr;
  size_t hcap = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

void resources_release(Resources* r) {
  if (r->device < 0) return;
  int cur = -1;
  cudaGetDevice(&cur);
  cudaSetDevice(r->device);
  if (r->stream) cudaStreamSynchronize(r->stream);
  if (r->dmem) cudaFree(r->dmem);
  if (r->hstage) cudaFreeHost(r->hstage);
  if (r->ev0) cudaEventDestroy(r->ev0);
  if (r->ev1) cudaEventDestroy(r->ev1);
  if (r->own_stream && r->stream) cudaStreamDestroy(r->stream);
  if (cur >= 0) cudaSetDevice(cur);
  *r = Resources();
}

ld_status resources_acquire(Resources* r, int device, cudaStream_t user_stream, size_t dbytes,
                            size_t hbytes) {
  LD_CUDA(cudaSetDevice(device));
  if (r->device < 0) {
    r->device = device;
    if (user_stream) { r->stream = user_stream; r->own_stream = false; }
    else { LD_CUDA(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking)); r->own_stream = true; }
    LD_CUDA(cudaEventCreate(&r->ev0));
    LD_CUDA(cudaEventCreate(&r->ev1));
  }
  if (r->dcap < dbytes) {
    if (r->dmem) { LD_CUDA(cudaStreamSynchronize(r->stream)); LD_CUDA(cudaFree(r->dmem)); r->dmem = nullptr; r->dcap = 0; }
    LD_CUDA(cudaMalloc(&r->dmem, dbytes));
    r->dcap = dbytes;
  }
  if (r->hcap < hbytes) {
    if (r->hstage) { LD_CUDA(cudaStreamSynchronize(r->stream)); LD_CUDA(cudaFreeHost(r->hstage)); r->hstage = nullptr; r->hcap = 0; }
    LD_CUDA(cudaMallocHost(&r->hstage, hbytes));
    r->hcap = hbytes;
  }
  return LD_OK;
}

std::mutex g_ws_mu[64];
Resources g_ws[64];

constexpr size_t kOffCounter = 0, kOffGvalue = 8, kOffResult = 16;
constexpr size_t kOffTot = 256, kOffH0 = 512, kOffA = 768;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

struct ld_plan {
  int device = 0;
  int R = 0, C = 0, d = 0, marginal = 0;
  Choice ch;
  Bounds bounds{};
  int k = 0, B = 1, fw = 0;                       // table geometry
  unsigned long long walk_len = 1, walks = 1, walk_begin = 0, walk_end = 1;
  unsigned long long n_begin = 0, n_end = 0;      // wide geometry
  unsigned long long total = 0;
  int blocks = 1, tpb = 128;
  size_t smem = 0;
  long long value_offset = 0;
  Resources own;
  Resources* res = nullptr;
  size_t upload_bytes = 0;
  bool uploaded = false;       // the upload belongs to the next fetched launch
  ld::Reduce red{};
  const void* kfn = nullptr;
  bool launched = false;
};

static void plan_free(ld_plan* p) {
  if (!p) return;
  if (p->res == &p->own) resources_release(&p->own);
  delete p;
}

extern "C" void ld_options_init(ld_options* o) {
  if (!o) return;
  memset(o, 0, sizeof *o);
  o->low_rows = -1;
  o->shard_count = 1;
}

extern "C" int ld_device_max_threads(int device, int* out) {
  DeviceInfo di;
  ld_status st = device_info(device, &di);
  if (st != LD_OK) return (int)st;
  *out = di.max_threads;
  return 0;
}

// Split [0, n) into `count` contiguous parts; part `idx` (calc_jmin_jmax form).
static void split_range(unsigned long long n, int idx, int count, unsigned long long* lo,
                        unsigned long long* hi) {
  if (count <= 1) { *lo = 0; *hi = n; return; }
  const unsigned long long c = (unsigned long long)count, i = (unsigned long long)idx;
  const unsigned long long q = n / c, r = n % c;
  *lo = i * q + (i < r ? i : r);
  *hi = *lo + q + (i < r ? 1ull : 0ull);
}

// Geometry, kernel choice and the upload image; resources are attached by
// the caller.  `shared` selects the per-device workspace instead of owned
// resources.
static ld_status plan_build(const int64_t* a, int R, int C, int d, int marginal, const ld_options* opt,
                            Resources* shared, ld_plan** out) {
  ld_options o;
  if (opt) o = *opt; else ld_options_init(&o);
  if (!a || R < 1 || C < 1) return ld_fail(LD_ERR_ARG, "empty matrix (%d x %d)", R, C);
  if (d < 1 || d > LD_MAX_D) return ld_fail(LD_ERR_ARG, "order d=%d outside 1..%d", d, LD_MAX_D);
  if (marginal && d != 1) return ld_fail(LD_ERR_ARG, "marginals need d == 1");
  if (C > LD_MAX_COLS) return ld_fail(LD_ERR_LIMIT, "%d columns exceed %d", C, LD_MAX_COLS);
  if (R > ld_max_rows_for(d)) return ld_fail(LD_ERR_LIMIT, "%d rows exceed %d for d=%d", R, ld_max_rows_for(d), d);
  if (o.shard_count < 0 || (o.shard_count > 1 && (o.shard_index < 0 || o.shard_index >= o.shard_count)))
    return ld_fail(LD_ERR_ARG, "shard %d of %d", o.shard_index, o.shard_count);
  const unsigned long long total = ld_labelings(R, d);
  if (total >= (1ull << 63)) return ld_fail(LD_ERR_LIMIT, "%d rows give 2^63 or more labelings", R);
  DeviceInfo di;
  ld_status st = device_info(o.device, &di);
  if (st != LD_OK) return st;
  if (cudaSetDevice(o.device) != cudaSuccess) return ld_fail(LD_ERR_CUDA, "cudaSetDevice(%d) failed", o.device);

  ld_plan* p = new ld_plan();
  p->device = o.device;
  p->R = R; p->C = C; p->d = d; p->marginal = marginal;
  p->total = total;
  p->bounds = compute_bounds(a, R, C, marginal);
  st = choose_kernel(R, C, d, marginal, p->bounds, o, &p->ch);
  if (st != LD_OK) { delete p; return st; }

  const int base = d <= 2 ? 2 : d;
  const int F = R - 1;
  std::vector<char> image;
  if (p->ch.kind == LD_KERNEL_TABLE) {
    const int D = p->ch.D, W = p->ch.W, PK = p->ch.PK, NW = D * W;
    p->kfn = ld::table_kernel_ptr(D, W, PK);
    if (!p->kfn) { delete p; return ld_fail(LD_ERR_ARG, "no table kernel for D=%d W=%d PK=%d", D, W, PK); }
    // low rows: largest k with base^k <= 1024 and a table of at most 32 KB
    const int maxB = std::min(1024, 8192 / NW);
    int k = 0;
    while (k < F && ipow(base, k + 1) <= (unsigned long long)maxB) ++k;
    if (o.low_rows >= 0 && o.low_rows <= F && ipow(base, o.low_rows) * NW <= 16384ull) k = o.low_rows;
    p->k = k;
    p->B = (int)ipow(base, k);
    p->tpb = ld::kTableThreads;
    p->smem = (size_t)ld::table_smem_words(D, W, R, p->B) * sizeof(uint32_t);
    if (cudaFuncSetAttribute(p->kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->smem) != cudaSuccess) {
      delete p; return ld_fail(LD_ERR_CUDA, "cannot reserve %zu bytes of shared memory", p->smem);
    }
    int bps = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, p->kfn, p->tpb, p->smem) != cudaSuccess || bps < 1) {
      delete p; return ld_fail(LD_ERR_CUDA, "table kernel does not fit an SM (smem %zu)", p->smem);
    }
    const unsigned long long full = (unsigned long long)di.sms * bps * p->tpb;
    const int nh = F - k;
    // walk length: as long as the walks still number >= 32 per thread of a full grid
    int fw = 0;
    while (fw < nh && ipow(base, nh - fw - 1) >= 32ull * full) ++fw;
    if (o.tile > 0) fw = std::min(nh, o.tile);
    p->fw = fw;
    p->walk_len = ipow(base, fw);
    p->walks = ipow(base, nh - fw);
    split_range(p->walks, o.shard_index, o.shard_count, &p->walk_begin, &p->walk_end);
    const unsigned long long mine = p->walk_end - p->walk_begin;
    const unsigned long long want = (mine + p->tpb - 1) / p->tpb;
    p->blocks = (int)std::min<unsigned long long>((unsigned long long)di.sms * bps, std::max(1ull, want));
    if (o.blocks > 0) p->blocks = o.blocks;
    // upload image: header | totals | initial H | packed rows
    std::vector<int64_t> tot(C, 0), h0(C, 0);
    for (int i = 0; i < R; ++i)
      for (int l = 0; l < C; ++l) tot[l] += a[(size_t)i * C + l];
    if (D == 1) {
      for (int l = 0; l < C; ++l) h0[l] = a[(size_t)(R - 1) * C + l];
      if (marginal) { h0[0] += p->bounds.K; p->value_offset = p->bounds.K; }
    }
    p->upload_bytes = kOffA + (size_t)R * W * 4;
    image.assign(p->upload_bytes, 0);
    pack_row(tot.data(), C, W, PK, (uint32_t*)(image.data() + kOffTot));
    pack_row(h0.data(), C, W, PK, (uint32_t*)(image.data() + kOffH0));
    for (int i = 0; i < R; ++i)
      pack_row(a + (size_t)i * C, C, W, PK, (uint32_t*)(image.data() + kOffA) + (size_t)i * W);
  } else {
    p->kfn = ld::wide_kernel_ptr(p->ch.i64, p->ch.PC, p->ch.multi);
    if (!p->kfn) { delete p; return ld_fail(LD_ERR_ARG, "no wide kernel for PC=%d", p->ch.PC); }
    p->tpb = ld::kWideThreads;
    int bps = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, p->kfn, p->tpb, 0) != cudaSuccess || bps < 1) bps = 1;
    split_range(total, o.shard_index, o.shard_count, &p->n_begin, &p->n_end);
    const unsigned long long mine = p->n_end - p->n_begin;
    const unsigned long long warps_full = (unsigned long long)di.sms * bps * (p->tpb / 32);
    const unsigned long long want_warps = std::max(1ull, std::min(warps_full, mine));
    p->blocks = (int)((want_warps + (p->tpb / 32) - 1) / (p->tpb / 32));
    if (o.blocks > 0) p->blocks = o.blocks;
    const size_t esz = p->ch.i64 ? 8 : 4;
    p->upload_bytes = kOffA + (size_t)R * C * esz;
    image.assign(p->upload_bytes, 0);
    if (p->ch.i64) memcpy(image.data() + kOffA, a, (size_t)R * C * 8);
    else {
      int32_t* dst = (int32_t*)(image.data() + kOffA);
      for (size_t t = 0; t < (size_t)R * C; ++t) dst[t] = (int32_t)a[t];
    }
  }
  // scratch header: counter 0, gvalue LLONG_MIN
  const long long gmin = LLONG_MIN;
  memcpy(image.data() + kOffGvalue, &gmin, sizeof gmin);

  const size_t off_slots = align256(p->upload_bytes);
  const size_t dbytes = off_slots + align256((size_t)p->blocks * sizeof(ld::Slot));
  p->res = shared ? shared : &p->own;
  st = resources_acquire(p->res, o.device, (cudaStream_t)o.stream, dbytes, p->upload_bytes);
  if (st != LD_OK) { plan_free(p); return st; }
  char* base_ptr = (char*)p->res->dmem;
  p->red.counter = (unsigned int*)(base_ptr + kOffCounter);
  p->red.gvalue = (long long*)(base_ptr + kOffGvalue);
  p->red.result = (ld::Slot*)(base_ptr + kOffResult);
  p->red.slots = (ld::Slot*)(base_ptr + off_slots);
  memcpy(p->res->hstage, image.data(), p->upload_bytes);
  cudaError_t ce = cudaMemcpyAsync(p->res->dmem, p->res->hstage, p->upload_bytes, cudaMemcpyHostToDevice,
                                   p->res->stream);
  if (ce == cudaSuccess && !shared) ce = cudaStreamSynchronize(p->res->stream);
  if (ce != cudaSuccess) { plan_free(p); return ld_fail(LD_ERR_CUDA, "upload failed: %s", cudaGetErrorString(ce)); }
  p->uploaded = true;
  *out = p;
  return LD_OK;
}

static ld_status plan_enqueue(ld_plan* p) {
  Resources* r = p->res;
  char* base_ptr = (char*)r->dmem;
  LD_CUDA(cudaSetDevice(p->device));
  LD_CUDA(cudaEventRecord(r->ev0, r->stream));
  if (p->ch.kind == LD_KERNEL_TABLE) {
    ld::TableArgs args;
    args.A = (const uint32_t*)(base_ptr + kOffA);
    args.tot = (const uint32_t*)(base_ptr + kOffTot);
    args.hinit = (const uint32_t*)(base_ptr + kOffH0);
    args.R = p->R; args.k = p->k; args.B = p->B; args.fw = p->fw;
    args.walk_len = p->walk_len; args.walk_begin = p->walk_begin; args.walk_end = p->walk_end;
    args.value_offset = p->value_offset;
    args.red = p->red;
    void* params[] = {&args};
    LD_CUDA(cudaLaunchKernel(p->kfn, dim3(p->blocks), dim3(p->tpb), params, p->smem, r->stream));
  } else if (p->ch.i64) {
    ld::WideArgs<long long> args;
    args.A = (const long long*)(base_ptr + kOffA);
    args.R = p->R; args.C = p->C; args.d = p->d; args.marginal = p->marginal;
    args.n_begin = p->n_begin; args.n_end = p->n_end;
    args.red = p->red;
    void* params[] = {&args};
    LD_CUDA(cudaLaunchKernel(p->kfn, dim3(p->blocks), dim3(p->tpb), params, 0, r->stream));
  } else {
    ld::WideArgs<int> args;
    args.A = (const int*)(base_ptr + kOffA);
    args.R = p->R; args.C = p->C; args.d = p->d; args.marginal = p->marginal;
    args.n_begin = p->n_begin; args.n_end = p->n_end;
    args.red = p->red;
    void* params[] = {&args};
    LD_CUDA(cudaLaunchKernel(p->kfn, dim3(p->blocks), dim3(p->tpb), params, 0, r->stream));
  }
  LD_CUDA(cudaEventRecord(r->ev1, r->stream));
  p->launched = true;
  return LD_OK;
}

static ld_status plan_fetch(ld_plan* p, ld_result* res, int32_t* strategy) {
  if (!p->launched) return ld_fail(LD_ERR_ARG, "plan has not been launched");
  Resources* r = p->res;
  LD_CUDA(cudaSetDevice(p->device));
  ld::Slot* h = (ld::Slot*)((char*)r->hstage + kOffResult);
  LD_CUDA(cudaMemcpyAsync(h, p->red.result, sizeof(ld::Slot), cudaMemcpyDeviceToHost, r->stream));
  LD_CUDA(cudaStreamSynchronize(r->stream));
  float ms = 0.f;
  LD_CUDA(cudaEventElapsedTime(&ms, r->ev0, r->ev1));
  memset(res, 0, sizeof *res);
  res->value = h->value;
  res->gray_index = h->index;
  res->labelings = p->ch.kind == LD_KERNEL_TABLE
                       ? (p->walk_end - p->walk_begin) * p->walk_len * (unsigned long long)p->B
                       : p->n_end - p->n_begin;
  res->kernel_ms = ms;
  res->kernel_kind = p->ch.kind;
  res->lane_bits = p->ch.lane_bits;
  res->h2d_bytes = p->uploaded ? p->upload_bytes : 0;
  res->d2h_bytes = sizeof(ld::Slot);
  if (strategy) ld_gray_labels(res->gray_index, p->R, p->d, strategy);
  p->uploaded = false;
  return LD_OK;
}

extern "C" ld_status ld_plan_create(const int64_t* a, int32_t rows, int32_t cols, int32_t d,
                                    int32_t marginal, const ld_options* opt, ld_plan** out) {
  if (!out) return ld_fail(LD_ERR_ARG, "null output");
  return plan_build(a, rows, cols, d, marginal, opt, nullptr, out);
}

extern "C" ld_status ld_plan_launch(ld_plan* plan) {
  if (!plan) return ld_fail(LD_ERR_ARG, "null plan");
  return plan_enqueue(plan);
}

extern "C" ld_status ld_plan_result(ld_plan* plan, ld_result* res, int32_t* strategy) {
  if (!plan || !res) return ld_fail(LD_ERR_ARG, "null argument");
  return plan_fetch(plan, res, strategy);
}

extern "C" ld_status ld_plan_range(const ld_plan* p, uint64_t* lo, uint64_t* hi) {
  if (!p || !lo || !hi) return ld_fail(LD_ERR_ARG, "null argument");
  if (p->ch.kind == LD_KERNEL_TABLE) {
    const unsigned long long span = p->walk_len * (unsigned long long)p->B;
    *lo = p->walk_begin * span;
    *hi = p->walk_end * span;
  } else {
    *lo = p->n_begin;
    *hi = p->n_end;
  }
  return LD_OK;
}

extern "C" ld_status ld_plan_describe(const ld_plan* p, char* buf, size_t cap) {
  if (!p || !buf) return ld_fail(LD_ERR_ARG, "null argument");
  if (p->ch.kind == LD_KERNEL_TABLE)
    snprintf(buf, cap,
             "table D=%d W=%d PK=%d (%d-bit lanes) k=%d B=%d fw=%d walks=%llu blocks=%d tpb=%d smem=%zu",
             p->ch.D, p->ch.W, p->ch.PK, p->ch.lane_bits, p->k, p->B, p->fw,
             (unsigned long long)p->walks, p->blocks, p->tpb, p->smem);
  else
    snprintf(buf, cap, "wide PC=%d multi=%d %s blocks=%d tpb=%d", p->ch.PC, p->ch.multi,
             p->ch.i64 ? "int64" : "int32", p->blocks, p->tpb);
  return LD_OK;
}

extern "C" void* ld_plan_stream(const ld_plan* p) { return p && p->res ? (void*)p->res->stream : nullptr; }

extern "C" void* ld_plan_result_device(const ld_plan* p) { return p ? (void*)p->red.result : nullptr; }

extern "C" void ld_plan_destroy(ld_plan* p) { plan_free(p); }

extern "C" ld_status ld_solve_reduced(const int64_t* a, int32_t rows, int32_t cols, int32_t d,
                                      int32_t marginal, const ld_options* opt, ld_result* res,
                                      int32_t* strategy) {
  if (!res) return ld_fail(LD_ERR_ARG, "null result");
  const int dev = opt ? opt->device : 0;
  if (dev < 0 || dev >= 64) return ld_fail(LD_ERR_ARG, "device %d out of range", dev);
  const bool use_ws = !(opt && opt->stream);
  std::unique_lock<std::mutex> lk(g_ws_mu[dev], std::defer_lock);
  if (use_ws) lk.lock();
  ld_plan* p = nullptr;
  ld_status st = plan_build(a, rows, cols, d, marginal, opt, use_ws ? &g_ws[dev] : nullptr, &p);
  if (st != LD_OK) return st;
  st = plan_enqueue(p);
  if (st == LD_OK) st = plan_fetch(p, res, strategy);
  plan_free(p);
  return st;
}
