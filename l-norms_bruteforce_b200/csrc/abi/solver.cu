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
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "smem_limit.h"
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
  int D = 0, WB = 0, WA = 0, WT = 0, k = 0;   // table: int32 words, int8x4 words, padded, low rows
  std::vector<int> order;                     // table: column of each lane (wide first)
  int PC = 0, multi = 0, i64 = 0;             // wide
  int lane_bits = 0;
  int lin = 0;                                // table: LM column 0 linear in word 0
  int pair = 0;                               // table: two high indices per thread
};

int round4(int x) { return (x + 3) & ~3; }

unsigned long long ipow(unsigned long long b, int e) {
  unsigned long long r = 1;
  for (int i = 0; i < e; ++i) r *= b;
  return r;
}

// Table-kernel configuration for a given number of low rows k: which columns
// can live in 8-bit lanes.  For d = 1 the two operands of each absolute
// difference are the high rows' partial sum (with the fixed row) and the low
// rows' partial sum, so each only needs its own part to fit 8 bits; for LM,
// column 0 carries the shift K split the same way (K_H + K_L).  For d >= 2 a
// table vector holds the column total minus low rows, so a column is narrow
// when its full bound fits.  Returns false if no instance exists.
bool table_config(const int64_t* a, int R, int C, int d, int marginal, int k, int force_bits,
                  Choice* ch) {
  std::vector<int> wide, narrow;
  for (int l = 0; l < C; ++l) {
    long long hb = 0, lb = 0;
    for (int i = 0; i < R; ++i) {
      const int64_t v = a[(size_t)i * C + l];
      const long long av = v < 0 ? -(long long)v : (long long)v;
      if (i < k) lb += av; else hb += av;
    }
    bool nar;
    if (d == 1) nar = (marginal && l == 0) ? (2 * hb <= 127 && 2 * lb <= 128) : (hb <= 127 && lb <= 127);
    else nar = hb + lb <= 127;
    if (force_bits == 32) nar = false;
    (nar ? narrow : wide).push_back(l);
  }
  if (force_bits == 8 && !wide.empty()) return false;
  int WB = (int)wide.size(), WA = ((int)narrow.size() + 3) / 4;
  if (d >= 2 && WB > 0 && WA > 0) {             // no mixed instances for d >= 2
    if (force_bits == 8) return false;
    wide.insert(wide.end(), narrow.begin(), narrow.end());
    narrow.clear();
    WB = C; WA = 0;
  }
  if (d >= 4 && WA == 0) WB = round4(WB);      // d >= 4: 32-bit instances come in multiples of 4 words
  if (!ld::table_kernel_mixed_ptr(d, WB, WA)) {
    if (force_bits == 8 || C > 64 || !ld::table_kernel_mixed_ptr(d, C, 0)) return false;
    wide.clear();
    for (int l = 0; l < C; ++l) wide.push_back(l);
    narrow.clear();
    WB = C; WA = 0;
  }
  ch->kind = LD_KERNEL_TABLE;
  ch->D = d; ch->WB = WB; ch->WA = WA; ch->WT = round4(WB + WA); ch->k = k;
  ch->order = wide;
  ch->order.insert(ch->order.end(), narrow.begin(), narrow.end());
  ch->lane_bits = WB > 0 ? 32 : 8;
  return true;
}

// Pick the kernel and, for the table kernel, the low-row count minimizing
// an estimate of the solve time: labelings x (words per labeling + the
// amortized cost of a high-row step) / threads that have work.
ld_status choose_kernel(const int64_t* a, int R, int C, int d, int marginal, const Bounds& b,
                        const ld_options& o, unsigned long long full_threads, Choice* ch) {
  if (b.overflow) return ld_fail(LD_ERR_LIMIT, "matrix entries too large: column sums exceed 2^61");
  const long long maxabs = std::max(b.colbound, marginal ? 2 * b.K : 0LL);
  const long long vmax = b.total + (marginal ? b.K : 0LL);
  const bool fits32 = vmax <= (long long)INT32_MAX && maxabs <= (long long)INT32_MAX;
  if (o.lane_bits && o.lane_bits != 8 && o.lane_bits != 32 && o.lane_bits != 64)
    return ld_fail(LD_ERR_ARG, "lane width %d is not 8, 32 or 64", o.lane_bits);
  if (o.kernel != LD_KERNEL_WIDE && d <= 10 && o.lane_bits != 64 && fits32) {
    const int base = d <= 2 ? 2 : d, F = R - 1;
    double best_t = 0;
    bool found = false;
    for (int k = 0; k <= F; ++k) {
      const unsigned long long B = ipow(base, k);
      if (B > 1024) break;
      if (o.low_rows >= 0 && k != std::min(o.low_rows, F)) continue;
      Choice c;
      if (!table_config(a, R, C, d, marginal, k, o.lane_bits, &c)) continue;
      const int NW = d * c.WT;
      if (B * (unsigned long long)NW > (o.low_rows >= 0 ? 16384ull : 8192ull)) continue;
      const double words = (double)d * (c.WB + c.WA);
      const double per_lab = words + (2.0 * words + 40.0) / (double)B;
      // parallel units: the high indices, or (d >= 3, label symmetry) the
      // ones that can hold a class minimum; time ~ units * B * per_lab
      // spread over min(units, threads)
      double units = (double)ipow(base, F - k);
      if (d >= 3 && !o.enumerate_all && F - k > 0) {
        uint64_t pass = 0;
        if (ld_symmetry_walks(d, F - k, 0, ipow(base, F - k), &pass) == LD_OK && pass > 0) units = (double)pass;
      }
      const double t = units * (double)B * per_lab / std::min(units, (double)full_threads);
      if (!found || t < best_t * 0.999) { best_t = t; *ch = c; found = true; }
    }
    if (found) return LD_OK;
    if (o.kernel == LD_KERNEL_TABLE)
      return ld_fail(LD_ERR_ARG, "the table kernel cannot take this matrix (d=%d, %d columns)", d, C);
  }
  if (o.kernel == LD_KERNEL_TABLE)
    return ld_fail(LD_ERR_ARG, "the table kernel cannot take this matrix (d=%d, %d columns)", d, C);
  if (o.lane_bits == 8) return ld_fail(LD_ERR_ARG, "8-bit lanes need the table kernel");
  ch->kind = LD_KERNEL_WIDE;
  ch->i64 = (!fits32 || o.lane_bits == 64) ? 1 : 0;
  ch->lane_bits = ch->i64 ? 64 : 32;
  int pc = 1;
  while (pc * 32 < C) pc *= 2;
  ch->PC = pc;
  ch->multi = d >= 2;
  return LD_OK;
}

// Pack one row into the kernel's words: WB int32 lanes (columns order[0..WB)),
// then WA words of four int8 lanes (the following columns), zero padded to WT.
void pack_row(const int64_t* row, const Choice& ch, uint32_t* out) {
  const int n = (int)ch.order.size();
  for (int w = 0; w < ch.WT; ++w) out[w] = 0u;
  for (int w = 0; w < ch.WB && w < n; ++w) out[w] = (uint32_t)(int32_t)row[ch.order[w]];
  for (int q = 0; q < ch.WA; ++q)
    for (int c = 0; c < 4; ++c) {
      const int p = ch.WB + 4 * q + c;
      if (p < n) out[ch.WB + q] |= ((uint32_t)(int32_t)row[ch.order[p]] & 0xffu) << (8 * c);
    }
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
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
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
  if (r->ev2) cudaEventDestroy(r->ev2);
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
    LD_CUDA(cudaEventCreate(&r->ev2));
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
// per-device workspace of the pruned search (its own stream, arena and
// pinned result staging), kept between calls
std::mutex g_pws_mu[64];
Resources g_pws[64];

constexpr size_t kOffCounter = 0, kOffGvalue = 8, kOffResult = 16;
constexpr size_t kOffTot = 256, kOffH0 = 512, kOffTb = 768, kOffA = 1024;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

struct ld_plan {
  int device = 0;
  int R = 0, C = 0, d = 0, marginal = 0;
  Choice ch;
  Bounds bounds{};
  int k = 0, B = 1, fw = 0;                       // table geometry
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
  st = choose_kernel(a, R, C, d, marginal, p->bounds, o, (unsigned long long)di.sms * 4 * 128, &p->ch);
  if (st != LD_OK) { delete p; return st; }

  const int base = d <= 2 ? 2 : d;
  const int F = R - 1;
  std::vector<char> image;
  if (p->ch.kind == LD_KERNEL_TABLE) {
    const int D = p->ch.D, WT = p->ch.WT;
    p->kfn = ld::table_kernel_mixed_ptr(D, p->ch.WB, p->ch.WA);
    if (!p->kfn) { delete p; return ld_fail(LD_ERR_ARG, "no table kernel for D=%d WB=%d WA=%d", D, p->ch.WB, p->ch.WA); }
    // LM with the marginal column in a 32-bit word of its own: its term is
    // never negative, so the instance that adds it linearly applies
    if (D == 1 && marginal && p->ch.WB >= 1 && !p->ch.order.empty() && p->ch.order[0] == 0) {
      if (const void* lk = ld::table_kernel_lin_ptr(p->ch.WB, p->ch.WA)) { p->kfn = lk; p->ch.lin = 1; }
    }
    const int k = p->ch.k;
    p->k = k;
    p->B = (int)ipow(base, k);
    p->tpb = ld::kTableThreads;
    p->smem = (size_t)ld::table_smem_words(D, WT, R, p->B) * sizeof(uint32_t);
    if (ld_raise_smem_limit(p->kfn, p->smem) != cudaSuccess) {
      delete p; return ld_fail(LD_ERR_CUDA, "cannot reserve %zu bytes of shared memory", p->smem);
    }
    int bps = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, p->kfn, p->tpb, p->smem) != cudaSuccess || bps < 1) {
      delete p; return ld_fail(LD_ERR_CUDA, "table kernel does not fit an SM (smem %zu)", p->smem);
    }
    const unsigned long long full = (unsigned long long)di.sms * bps * p->tpb;
    const int nh = F - k;
    // d >= 3: walks that hold no smallest index of a label-permutation
    // class are skipped (symmetry.c); the walks that run decide the length
    const bool sym = D >= 3 && !o.enumerate_all;
    auto walks_run = [&](int f, unsigned long long lo, unsigned long long hi) -> unsigned long long {
      uint64_t c = hi - lo;
      if (sym && nh - f > 0 && ld_symmetry_walks(d, nh - f, lo, hi, &c) != LD_OK) c = hi - lo;
      return (unsigned long long)c;
    };
    // walk length: as long as the walks still number >= 32 per thread of a
    // full grid (d <= 2), or >= 4 (d >= 3, whose walk seeding costs 64-bit
    // divisions per high digit: longer walks measured 9 % faster on 20x30
    // d = 3)
    const unsigned long long per_thread = D >= 3 ? 4ull : 32ull;
    int fw = 0;
    while (fw < nh && walks_run(fw + 1, 0, ipow(base, nh - fw - 1)) >= per_thread * full) ++fw;
    if (o.tile > 0) fw = std::min(nh, o.tile);
    p->fw = fw;
    p->walk_len = ipow(base, fw);
    p->walks = ipow(base, nh - fw);
    if (sym && nh - fw > 0) p->sym_digits = nh - fw;
    if (p->sym_digits > 0 && o.shard_count > 1) {
      // shards of equal work: equal numbers of walks that pass
      uint64_t lo = 0, hi = 0;
      const ld_status sst = ld_sym_split(d, p->sym_digits, o.shard_index, o.shard_count, &lo, &hi);
      if (sst != LD_OK) { delete p; return sst; }
      p->walk_begin = lo; p->walk_end = hi;
    } else {
      split_range(p->walks, o.shard_index, o.shard_count, &p->walk_begin, &p->walk_end);
    }
    p->walks_run = walks_run(fw, p->walk_begin, p->walk_end);
    if (p->sym_digits > 0) {
      p->rank_begin = walks_run(fw, 0, p->walk_begin);
      p->rank_end = p->rank_begin + p->walks_run;
    }
    const unsigned long long mine = p->walks_run;
    const unsigned long long want = (mine + p->tpb - 1) / p->tpb;
    p->blocks = (int)std::min<unsigned long long>((unsigned long long)di.sms * bps, std::max(1ull, want));
    if (o.blocks > 0) p->blocks = o.blocks;
    // at least two walks per thread: the instance that walks two high
    // indices per thread against each table entry read (L_1 / LM, <= 10 words)
    if (D == 1 && mine >= 2ull * (unsigned long long)p->blocks * (unsigned long long)p->tpb) {
      const void* pk = ld::table_kernel_pair_ptr(p->ch.WB, p->ch.WA, p->ch.lin);
      int pbps = 0;
      if (pk && ld_raise_smem_limit(pk, p->smem) == cudaSuccess &&
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pbps, pk, p->tpb, p->smem) == cudaSuccess && pbps >= 1) {
        p->kfn = pk;
        p->ch.pair = 1;
        if (o.blocks <= 0)
          p->blocks = (int)std::min<unsigned long long>((unsigned long long)di.sms * pbps, std::max(1ull, want));
      }
    }
    // upload image: header | totals | initial H | table bias | packed rows
    std::vector<int64_t> tot(C, 0), h0(C, 0), tb(C, 0);
    for (int i = 0; i < R; ++i)
      for (int l = 0; l < C; ++l) tot[l] += a[(size_t)i * C + l];
    if (D == 1) {
      for (int l = 0; l < C; ++l) h0[l] = a[(size_t)(R - 1) * C + l];
      if (marginal) {
        long long kl = 0, kh = 0;   // the low rows' and the other rows' share of K
        for (int i = 0; i < R; ++i) {
          const int64_t v = a[(size_t)i * C];
          (i < k ? kl : kh) += v < 0 ? -(long long)v : (long long)v;
        }
        h0[0] += kh;
        tb[0] = -kl;
        p->value_offset = kh + kl;
      }
    }
    p->upload_bytes = kOffA + (size_t)R * WT * 4;
    if (p->sym_digits > 0) {   // completion counts for handing out walks by rank
      p->sym_off = align256(p->upload_bytes);
      p->upload_bytes = p->sym_off + ld_sym_table_len(d, p->sym_digits) * sizeof(uint64_t);
    }
    image.assign(p->upload_bytes, 0);
    if (p->sym_digits > 0) {
      const ld_status sst = ld_sym_table(d, p->sym_digits, (uint64_t*)(image.data() + p->sym_off));
      if (sst != LD_OK) { delete p; return sst; }
    }
    pack_row(tot.data(), p->ch, (uint32_t*)(image.data() + kOffTot));
    pack_row(h0.data(), p->ch, (uint32_t*)(image.data() + kOffH0));
    pack_row(tb.data(), p->ch, (uint32_t*)(image.data() + kOffTb));
    for (int i = 0; i < R; ++i)
      pack_row(a + (size_t)i * C, p->ch, (uint32_t*)(image.data() + kOffA) + (size_t)i * WT);
  } else {
    p->kfn = ld::wide_kernel_ptr(p->ch.i64, p->ch.PC, p->ch.multi, 0);
    if (!p->kfn) { delete p; return ld_fail(LD_ERR_ARG, "no wide kernel for PC=%d", p->ch.PC); }
    p->tpb = ld::kWideThreads;
    int bps = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, p->kfn, p->tpb, 0) != cudaSuccess || bps < 1) bps = 1;
    const unsigned long long warps_full = (unsigned long long)di.sms * bps * (p->tpb / 32);
    // d >= 3: label symmetry over walks of d^L consecutive indices, handed
    // to warps by rank.  A walk costs a re-seed (R rows) plus its d^L steps;
    // the slowest warp takes ceil(passing walks / warps) of them.  The walk
    // length that minimises that estimate is used when it beats evaluating
    // every index (ceil(labelings / warps) steps plus one seed per warp).
    // Walks longer than 64 R indices no longer shorten the estimate.
    int L = -1;
    if (d >= 3 && !o.enumerate_all && F >= 2) {
      double best_t = (double)((total + warps_full - 1) / warps_full) + (double)R;
      for (int l = 0; l <= F - 1 && ipow(d, l) <= 64ull * (unsigned long long)R; ++l) {
        uint64_t k = 0;
        if (ld_symmetry_walks(d, F - l, 0, ipow(d, F - l), &k) != LD_OK || k == 0) continue;
        const double t = std::ceil((double)k / (double)warps_full) * ((double)R + (double)ipow(d, l));
        if (t < best_t) { best_t = t; L = l; }
      }
    }
    unsigned long long mine = 0;
    if (L >= 0) {
      const int P = F - L;
      p->kfn = ld::wide_kernel_ptr(p->ch.i64, p->ch.PC, p->ch.multi, 1);
      if (!p->kfn) { delete p; return ld_fail(LD_ERR_ARG, "no symmetric wide kernel for PC=%d", p->ch.PC); }
      p->sym_digits = P;
      p->walk_len = ipow(d, L);
      p->walks = ipow(d, P);
      uint64_t wb = 0, we = p->walks;
      if (o.shard_count > 1) {
        const ld_status sst = ld_sym_split(d, P, o.shard_index, o.shard_count, &wb, &we);
        if (sst != LD_OK) { delete p; return sst; }
      }
      uint64_t below = 0, run = 0;
      if (ld_symmetry_walks(d, P, 0, wb, &below) != LD_OK || ld_symmetry_walks(d, P, wb, we, &run) != LD_OK) {
        delete p; return ld_fail(LD_ERR_ARG, "symmetry count failed");
      }
      p->walk_begin = wb; p->walk_end = we;
      p->rank_begin = below; p->rank_end = below + run;
      p->walks_run = run;
      p->n_begin = wb * p->walk_len;
      p->n_end = we * p->walk_len;
      mine = run;
    } else {
      split_range(total, o.shard_index, o.shard_count, &p->n_begin, &p->n_end);
      mine = p->n_end - p->n_begin;
    }
    const unsigned long long want_warps = std::max(1ull, std::min(warps_full, mine));
    p->blocks = (int)((want_warps + (p->tpb / 32) - 1) / (p->tpb / 32));
    if (o.blocks > 0) p->blocks = o.blocks;
    const size_t esz = p->ch.i64 ? 8 : 4;
    p->upload_bytes = kOffA + (size_t)R * C * esz;
    if (p->sym_digits > 0) {   // completion counts for handing out walks by rank
      p->sym_off = align256(p->upload_bytes);
      p->upload_bytes = p->sym_off + ld_sym_table_len(d, p->sym_digits) * sizeof(uint64_t);
    }
    image.assign(p->upload_bytes, 0);
    if (p->ch.i64) memcpy(image.data() + kOffA, a, (size_t)R * C * 8);
    else {
      int32_t* dst = (int32_t*)(image.data() + kOffA);
      for (size_t t = 0; t < (size_t)R * C; ++t) dst[t] = (int32_t)a[t];
    }
    if (p->sym_digits > 0) {
      const ld_status sst = ld_sym_table(d, p->sym_digits, (uint64_t*)(image.data() + p->sym_off));
      if (sst != LD_OK) { delete p; return sst; }
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
    args.tbias = (const uint32_t*)(base_ptr + kOffTb);
    args.R = p->R; args.k = p->k; args.B = p->B; args.fw = p->fw;
    args.walk_len = p->walk_len; args.walk_begin = p->walk_begin; args.walk_end = p->walk_end;
    args.sym_digits = p->sym_digits;
    args.sym_table = (const unsigned long long*)(base_ptr + p->sym_off);
    args.rank_begin = p->rank_begin; args.rank_end = p->rank_end;
    args.value_offset = p->value_offset;
    args.red = p->red;
    void* params[] = {&args};
    LD_CUDA(cudaLaunchKernel(p->kfn, dim3(p->blocks), dim3(p->tpb), params, p->smem, r->stream));
  } else if (p->ch.i64) {
    ld::WideArgs<long long> args;
    args.A = (const long long*)(base_ptr + kOffA);
    args.R = p->R; args.C = p->C; args.d = p->d; args.marginal = p->marginal;
    args.n_begin = p->n_begin; args.n_end = p->n_end;
    args.sym_digits = p->sym_digits; args.walk_len = p->walk_len;
    args.sym_table = (const unsigned long long*)(base_ptr + p->sym_off);
    args.rank_begin = p->rank_begin; args.rank_end = p->rank_end;
    args.red = p->red;
    void* params[] = {&args};
    LD_CUDA(cudaLaunchKernel(p->kfn, dim3(p->blocks), dim3(p->tpb), params, 0, r->stream));
  } else {
    ld::WideArgs<int> args;
    args.A = (const int*)(base_ptr + kOffA);
    args.R = p->R; args.C = p->C; args.d = p->d; args.marginal = p->marginal;
    args.n_begin = p->n_begin; args.n_end = p->n_end;
    args.sym_digits = p->sym_digits; args.walk_len = p->walk_len;
    args.sym_table = (const unsigned long long*)(base_ptr + p->sym_off);
    args.rank_begin = p->rank_begin; args.rank_end = p->rank_end;
    args.red = p->red;
    void* params[] = {&args};
    LD_CUDA(cudaLaunchKernel(p->kfn, dim3(p->blocks), dim3(p->tpb), params, 0, r->stream));
  }
  LD_CUDA(cudaEventRecord(r->ev1, r->stream));
  p->launched = true;
  return LD_OK;
}

// labelings the plan's kernel computes a value for
static unsigned long long plan_evaluated(const ld_plan* p) {
  if (p->ch.kind == LD_KERNEL_TABLE) return p->walks_run * p->walk_len * (unsigned long long)p->B;
  if (p->ch.kind == LD_KERNEL_WIDE)
    return p->sym_digits > 0 ? p->walks_run * p->walk_len : p->n_end - p->n_begin;
  return 0;
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
  res->evaluated = plan_evaluated(p);
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
             "table D=%d int32 words=%d int8x4 words=%d lin=%d pair=%d k=%d B=%d fw=%d walks=%llu run=%llu "
             "sym=%d blocks=%d tpb=%d smem=%zu",
             p->ch.D, p->ch.WB, p->ch.WA, p->ch.lin, p->ch.pair, p->k, p->B, p->fw,
             (unsigned long long)p->walks, (unsigned long long)p->walks_run, p->sym_digits, p->blocks, p->tpb,
             p->smem);
  else
    snprintf(buf, cap, "wide PC=%d multi=%d %s blocks=%d tpb=%d sym=%d walk_len=%llu run=%llu", p->ch.PC,
             p->ch.multi, p->ch.i64 ? "int64" : "int32", p->blocks, p->tpb, p->sym_digits,
             (unsigned long long)p->walk_len, (unsigned long long)p->walks_run);
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

// ---------------------------------------------------------------------------
// Resumable solves: the shards of one solve run one after another, with a
// checkpoint after each (no counterpart in the reference, whose runs cannot
// be interrupted and resumed).
namespace {

// FNV-1a over the problem and the split, so that a checkpoint is only ever
// continued by the solve that wrote it
unsigned long long checkpoint_fingerprint(const int64_t* a, int R, int C, int d, int marginal, int pieces,
                                          int enumerate_all) {
  unsigned long long h = 1469598103934665603ull;
  auto mix = [&](const void* p, size_t n) {
    const unsigned char* c = (const unsigned char*)p;
    for (size_t i = 0; i < n; ++i) { h ^= c[i]; h *= 1099511628211ull; }
  };
  const int hdr[6] = {R, C, d, marginal, pieces, enumerate_all};
  mix(hdr, sizeof hdr);
  mix(a, (size_t)R * C * sizeof(int64_t));
  return h;
}

struct Checkpoint {
  unsigned long long fingerprint = 0;
  int pieces = 0, next = 0;
  unsigned long long covered = 0;             // Gray indices [0, covered) are done
  long long value = LLONG_MIN;                // best so far (LLONG_MIN: none)
  unsigned long long index = ULLONG_MAX;
  unsigned long long labelings = 0, evaluated = 0;
  double kernel_ms = 0;
};

// 1 = read, 0 = no file, -1 = unreadable
int checkpoint_read(const char* path, Checkpoint* ck) {
  FILE* f = fopen(path, "r");
  if (!f) return 0;
  int version = 0;
  const int n = fscanf(f, "lnorms-checkpoint %d fingerprint %llx pieces %d next %d covered %llu value %lld index %llu "
                          "labelings %llu evaluated %llu kernel_ms %lf",
                       &version, &ck->fingerprint, &ck->pieces, &ck->next, &ck->covered, &ck->value, &ck->index,
                       &ck->labelings, &ck->evaluated, &ck->kernel_ms);
  fclose(f);
  return (n == 10 && version == 1) ? 1 : -1;
}

bool checkpoint_write(const char* path, const Checkpoint& ck) {
  const std::string tmp = std::string(path) + ".tmp";
  FILE* f = fopen(tmp.c_str(), "w");
  if (!f) return false;
  const int n = fprintf(f,
                        "lnorms-checkpoint 1\nfingerprint %016llx\npieces %d\nnext %d\ncovered %llu\nvalue %lld\n"
                        "index %llu\nlabelings %llu\nevaluated %llu\nkernel_ms %.6f\n",
                        ck.fingerprint, ck.pieces, ck.next, ck.covered, ck.value, ck.index, ck.labelings,
                        ck.evaluated, ck.kernel_ms);
  const bool ok = n > 0 && fflush(f) == 0;
  if (fclose(f) != 0 || !ok) return false;
  return rename(tmp.c_str(), path) == 0;   // the old checkpoint stays valid until here
}

}  // namespace

extern "C" ld_status ld_solve_resumable(const int64_t* a, int32_t rows, int32_t cols, int32_t d, int32_t marginal,
                                        const ld_options* opt, int32_t pieces, const char* checkpoint_path,
                                        int32_t max_pieces, int32_t* done, ld_result* res, int32_t* strategy) {
  if (!a || !checkpoint_path || !done || !res) return ld_fail(LD_ERR_ARG, "null argument");
  if (rows < 1 || cols < 1 || d < 1 || d > LD_MAX_D) return ld_fail(LD_ERR_ARG, "bad problem %d x %d, d=%d", rows, cols, d);
  if (pieces < 1) return ld_fail(LD_ERR_ARG, "pieces must be >= 1 (got %d)", pieces);
  ld_options o;
  if (opt) o = *opt; else ld_options_init(&o);
  if (o.shard_count > 1) return ld_fail(LD_ERR_ARG, "a resumable solve makes its own shards");
  const int marg = d == 1 && marginal ? 1 : 0;
  const unsigned long long fp = checkpoint_fingerprint(a, rows, cols, d, marg, pieces, o.enumerate_all ? 1 : 0);
  Checkpoint ck;
  const int got = checkpoint_read(checkpoint_path, &ck);
  if (got < 0) return ld_fail(LD_ERR_IO, "%s is not a checkpoint of this library", checkpoint_path);
  if (got == 0) {
    ck = Checkpoint();
    ck.fingerprint = fp;
    ck.pieces = pieces;
  } else if (ck.fingerprint != fp || ck.pieces != pieces) {
    return ld_fail(LD_ERR_ARG, "%s belongs to another problem or split (fingerprint %016llx, %d pieces)",
                   checkpoint_path, ck.fingerprint, ck.pieces);
  } else if (ck.next < 0 || ck.next > pieces) {
    return ld_fail(LD_ERR_IO, "%s records piece %d of %d", checkpoint_path, ck.next, pieces);
  }
  int ran = 0;
  int kind = LD_KERNEL_NONE, lane_bits = 0;
  while (ck.next < pieces && (max_pieces <= 0 || ran < max_pieces)) {
    ld_options po = o;
    po.shard_index = ck.next;
    po.shard_count = pieces;
    ld_plan* p = nullptr;
    ld_status st = ld_plan_create(a, rows, cols, d, marg, &po, &p);
    if (st != LD_OK) return st;
    uint64_t lo = 0, hi = 0;
    ld_plan_range(p, &lo, &hi);
    if (pieces > 1 && lo != ck.covered) {
      ld_plan_destroy(p);
      return ld_fail(LD_ERR_ARG, "piece %d starts at Gray index %llu, the checkpoint covers [0, %llu): the solve's "
                     "geometry changed (options or device)", ck.next, (unsigned long long)lo, ck.covered);
    }
    ld_result r;
    st = ld_plan_launch(p);
    if (st == LD_OK) st = ld_plan_result(p, &r, nullptr);
    ld_plan_destroy(p);
    if (st != LD_OK) return st;
    if (r.value > ck.value || (r.value == ck.value && r.gray_index < ck.index)) {
      ck.value = r.value;
      ck.index = r.gray_index;
    }
    ck.covered = hi;
    ck.labelings += r.labelings;
    ck.evaluated += r.evaluated;
    ck.kernel_ms += r.kernel_ms;
    kind = r.kernel_kind;
    lane_bits = r.lane_bits;
    ++ck.next;
    ++ran;
    if (!checkpoint_write(checkpoint_path, ck)) return ld_fail(LD_ERR_IO, "cannot write %s", checkpoint_path);
  }
  *done = ck.next == pieces ? 1 : 0;
  memset(res, 0, sizeof *res);
  res->value = ck.value;
  res->gray_index = ck.index;
  res->labelings = ck.labelings;
  res->evaluated = ck.evaluated;
  res->kernel_ms = (float)ck.kernel_ms;
  res->kernel_kind = kind;
  res->lane_bits = lane_bits;
  if (*done && strategy) ld_gray_labels(ck.index, rows, d, strategy);
  return LD_OK;
}

// ---------------------------------------------------------------------------
// Pruned exact search (prune_kernel.cuh).  Exactly the plain enumeration's
// result; the incumbent only decides how much is skipped.
#include "../kernels/prune_kernel.cuh"

namespace {

// value of one labeling (labels of rows 0..R-2), int64
long long labeling_value(const int64_t* a, int R, int C, int d, int marginal, const int32_t* lab) {
  const int nm = d == 1 ? 1 : d;
  std::vector<long long> s((size_t)nm * C, 0);
  for (int l = 0; l < C; ++l) s[l] = a[(size_t)(R - 1) * C + l];
  for (int i = 0; i < R - 1; ++i)
    for (int l = 0; l < C; ++l) {
      const long long x = a[(size_t)i * C + l];
      if (d == 1) s[l] += lab[i] ? x : -x;
      else s[(size_t)lab[i] * C + l] += x;
    }
  long long v = 0;
  for (int m = 0; m < nm; ++m)
    for (int l = 0; l < C; ++l) {
      const long long x = s[(size_t)m * C + l];
      v += (d == 1 && marginal && l == 0) ? x : (x < 0 ? -x : x);
    }
  return v;
}

// The norm of rows [0, r) alone (every labeling of them), for the bounds:
// the plain solver on those rows plus a zero fixed row.  Falls back to the
// always-valid sum of absolute entries when the submatrix is too large to
// enumerate quickly.
ld_status rest_norm(const int64_t* a, int C, int d, int marginal, int r, int device, long long* out) {
  if (r <= 0) { *out = 0; return LD_OK; }
  const int base = d <= 2 ? 2 : d;
  if ((double)r * std::log2((double)base) > 34.0) {
    long long s = 0;
    for (int i = 0; i < r; ++i)
      for (int l = 0; l < C; ++l) { const int64_t x = a[(size_t)i * C + l]; s += x < 0 ? -x : x; }
    *out = s;
    return LD_OK;
  }
  std::vector<int64_t> sub((size_t)(r + 1) * C, 0);
  memcpy(sub.data(), a, sizeof(int64_t) * (size_t)r * C);
  ld_options o;
  ld_options_init(&o);
  o.device = device;
  ld_result res;
  ld_status st = ld_solve_reduced(sub.data(), r + 1, C, d, marginal, &o, &res, nullptr);
  if (st != LD_OK) return st;
  *out = res.value;
  return LD_OK;
}

}  // namespace

extern "C" ld_status ld_solve_pruned(const int64_t* a, int32_t R, int32_t C, int32_t d, int32_t marginal,
                                     const ld_options* opt, const int32_t* incumbent_labels,
                                     ld_result* res, int32_t* strategy, ld_prune_stats* stats) {
  if (!a || !res || R < 1 || C < 1) return ld_fail(LD_ERR_ARG, "bad arguments");
  ld_options o;
  if (opt) o = *opt; else ld_options_init(&o);
  ld_prune_stats ps;
  memset(&ps, 0, sizeof ps);
  ps.incumbent = LLONG_MIN;
  if (incumbent_labels && R > 1) {
    for (int i = 0; i < R - 1; ++i)
      if (incumbent_labels[i] < 0 || incumbent_labels[i] >= (d == 1 ? 2 : d))
        return ld_fail(LD_ERR_ARG, "incumbent label %d of row %d out of range", incumbent_labels[i], i);
    ps.incumbent = labeling_value(a, R, C, d, marginal, incumbent_labels);
  }
  auto plain = [&]() -> ld_status {
    ld_status s = ld_solve_reduced(a, R, C, d, marginal, &o, res, strategy);
    ps.pruned = 0;
    if (stats) *stats = ps;
    return s;
  };
  if (d > 3 || R < 3 || C > LD_MAX_COLS || R > ld_max_rows_for(d)) return plain();
  DeviceInfo di;
  ld_status st = device_info(o.device, &di);
  if (st != LD_OK) return st;
  const Bounds bnd = compute_bounds(a, R, C, marginal);
  if (bnd.overflow || bnd.total + (marginal ? bnd.K : 0) > (long long)INT32_MAX) return plain();

  // table configuration with a pruned-kernel instance: the largest k whose
  // table fits 48 KB
  const int base = d <= 2 ? 2 : d, F = R - 1;
  Choice ch;
  const void* kb = nullptr;
  const void* ks = nullptr;
  int k = -1;
  for (int kk = std::min(F - 1, 10); kk >= 0 && k < 0; --kk) {
    const unsigned long long B = ipow(base, kk);
    if (B > 1024) continue;
    Choice c;
    if (!table_config(a, R, C, d, marginal, kk, 0, &c)) continue;
    // round to an instantiated shape
    if (d == 1 && !(c.WB <= 2 && c.WA <= 16)) {
      if (C > 64) continue;
      c.order.clear();
      for (int l = 0; l < C; ++l) c.order.push_back(l);
      c.WB = round4(C); c.WA = 0; c.lane_bits = 32;
    } else if (d >= 2) {
      if (c.WA > 0) c.WA = round4(c.WA); else c.WB = round4(c.WB);
    }
    c.WT = round4(c.WB + c.WA);
    const void* b1; const void* b2;
    ld::prune_kernel_ptrs(d, c.WB, c.WA, &b1, &b2);
    if (!b1 || B * (unsigned long long)(d * c.WT) * 4ull > 48ull * 1024ull) continue;
    ch = c; kb = b1; ks = b2; k = kk;
  }
  if (k < 0) return plain();
  const int nh = F - k;
  // walk rows: every walk gets one bound in the first launch, so at most
  // about 2^21 walks; the surviving walks' high indices are split over the
  // threads of the scan, so long walks cost nothing extra there
  int fw = std::min(nh, 5);
  while (fw < nh && (double)(nh - fw) * std::log2((double)base) > 21.0) ++fw;
  const unsigned long long walk_len = ipow(base, fw), walks = ipow(base, nh - fw);
  const int B = (int)ipow(base, k);
  ps.low_rows = k; ps.walk_rows = fw;
  ps.walks_total = walks;
  ps.highs_total = walks * walk_len;
  ps.block = (uint64_t)B;

  // bounds of the rest rows, in the kernel's representation
  long long m_low = 0, m_walk = 0, kl = 0, kh = 0;
  st = rest_norm(a, C, d, marginal, k, o.device, &m_low);
  if (st == LD_OK) st = rest_norm(a, C, d, marginal, k + fw, o.device, &m_walk);
  if (st != LD_OK) return st;
  if (d == 1 && marginal) {
    for (int i = 0; i < R; ++i) { const int64_t v = a[(size_t)i * C]; (i < k ? kl : kh) += v < 0 ? -v : v; }
    m_low += kl;
    m_walk += kl;
  }
  const long long offset = kh + kl;
  const long long thr = ps.incumbent == LLONG_MIN ? LLONG_MIN : ps.incumbent + offset;

  // image: header | tot | h0 | tb | ttop | thigh | rows
  const int WT = ch.WT;
  std::vector<int64_t> tot(C, 0), h0(C, 0), tb(C, 0), ttop(C, 0), thigh(C, 0);
  for (int i = 0; i < R; ++i)
    for (int l = 0; l < C; ++l) {
      const int64_t x = a[(size_t)i * C + l];
      tot[l] += x;
      if (i >= k) thigh[l] += x;
      if (i >= k + fw) ttop[l] += x;
    }
  if (d == 1) {
    for (int l = 0; l < C; ++l) h0[l] = a[(size_t)(R - 1) * C + l];
    if (marginal) { h0[0] += kh; tb[0] = -kl; }
  }
  const size_t offTot = 256, offH0 = 512, offTb = 768, offTtop = 1024, offThigh = 1280, offA = 1536;
  const size_t upload = offA + (size_t)R * WT * 4;
  std::vector<char> image(upload, 0);
  const long long gmin = LLONG_MIN;
  memcpy(image.data() + 8, &gmin, sizeof gmin);
  pack_row(tot.data(), ch, (uint32_t*)(image.data() + offTot));
  pack_row(h0.data(), ch, (uint32_t*)(image.data() + offH0));
  pack_row(tb.data(), ch, (uint32_t*)(image.data() + offTb));
  pack_row(ttop.data(), ch, (uint32_t*)(image.data() + offTtop));
  pack_row(thigh.data(), ch, (uint32_t*)(image.data() + offThigh));
  for (int i = 0; i < R; ++i) pack_row(a + (size_t)i * C, ch, (uint32_t*)(image.data() + offA) + (size_t)i * WT);

  const size_t smem_b = (size_t)ld::prune_smem_words(d, WT, R, B, false) * 4;
  const size_t smem_s = (size_t)ld::prune_smem_words(d, WT, R, B, true) * 4;
  int bps_b = 0, bps_s = 0;
  if (cudaSetDevice(o.device) != cudaSuccess ||
      ld_raise_smem_limit(kb, smem_b) != cudaSuccess || ld_raise_smem_limit(ks, smem_s) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps_b, kb, ld::kPruneThreads, smem_b) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps_s, ks, ld::kPruneThreads, smem_s) != cudaSuccess ||
      bps_b < 1 || bps_s < 1)
    return ld_fail(LD_ERR_CUDA, "pruned kernels do not fit an SM");
  const unsigned long long blocks_b = std::max(1ull, std::min<unsigned long long>((unsigned long long)di.sms * bps_b,
                                                   (walks + ld::kPruneThreads - 1) / ld::kPruneThreads));
  const unsigned long long blocks_s = (unsigned long long)di.sms * bps_s;
  const size_t off_slots = align256(upload);
  const size_t off_list = off_slots + align256(blocks_s * sizeof(ld::Slot));
  const size_t off_cnt = off_list + align256(walks * 8);
  const size_t dbytes = off_cnt + 256;
  if (o.device < 0 || o.device >= 64) return ld_fail(LD_ERR_ARG, "device %d out of range", o.device);
  std::lock_guard<std::mutex> lock(g_pws_mu[o.device]);
  Resources* r = &g_pws[o.device];
  // the workspace keeps the stream it was created with: the caller's, or its own
  if (r->device >= 0 && (cudaStream_t)o.stream != (r->own_stream ? nullptr : r->stream)) resources_release(r);
  st = resources_acquire(r, o.device, (cudaStream_t)o.stream, dbytes, 256);
  if (st != LD_OK) return st;
  char* dmem = (char*)r->dmem;
  cudaStream_t s = r->stream;
  ld::Slot* out_h = (ld::Slot*)r->hstage;
  unsigned long long* hstat = (unsigned long long*)((char*)r->hstage + 64);
  float ms_b = 0.f, ms_s = 0.f;
  auto fail = [&](const char* what, cudaError_t e) {
    cudaStreamSynchronize(s);
    return ld_fail(LD_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  };
  cudaError_t e;
  if ((e = cudaMemsetAsync(dmem + off_cnt, 0, 256, s)) != cudaSuccess) return fail("memset", e);
  if ((e = cudaMemcpyAsync(dmem, image.data(), upload, cudaMemcpyHostToDevice, s)) != cudaSuccess) return fail("upload", e);
  {
    ld::PruneArgs args;
    ld::TableArgs& t = args.t;
    t.A = (const uint32_t*)(dmem + offA);
    t.tot = (const uint32_t*)(dmem + offTot);
    t.hinit = (const uint32_t*)(dmem + offH0);
    t.tbias = (const uint32_t*)(dmem + offTb);
    t.R = R; t.k = k; t.B = B; t.fw = fw;
    t.walk_len = walk_len; t.walk_begin = 0; t.walk_end = walks;
    // d = 3: the walk bound also drops walks that hold no class minimum
    t.sym_digits = (d == 3 && !o.enumerate_all && nh - fw > 0) ? nh - fw : 0;
    t.sym_table = nullptr; t.rank_begin = t.rank_end = 0;
    t.value_offset = offset;
    t.red.counter = (unsigned int*)(dmem + 0);
    t.red.gvalue = (long long*)(dmem + 8);
    t.red.result = (ld::Slot*)(dmem + 16);
    t.red.slots = (ld::Slot*)(dmem + off_slots);
    args.ttop = (const uint32_t*)(dmem + offTtop);
    args.thigh = (const uint32_t*)(dmem + offThigh);
    args.threshold = thr;
    args.m_walk = m_walk;
    args.m_low = m_low;
    args.list = (unsigned long long*)(dmem + off_list);
    args.list_count = (unsigned long long*)(dmem + off_cnt);
    args.stats = (unsigned long long*)(dmem + off_cnt + 8);
    void* params[] = {&args};
    if ((e = cudaEventRecord(r->ev0, s)) != cudaSuccess) return fail("event", e);
    if ((e = cudaLaunchKernel(kb, dim3((unsigned)blocks_b), dim3(ld::kPruneThreads), params, smem_b, s)) != cudaSuccess)
      return fail("walk bound launch", e);
    if ((e = cudaEventRecord(r->ev1, s)) != cudaSuccess) return fail("event", e);
    // When more than a quarter of the walks survive their bound the scan
    // would do most of the plain enumeration's work at a lower rate: run the
    // plain enumeration instead (same result).
    if ((e = cudaMemcpyAsync(hstat, dmem + off_cnt, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s)) !=
        cudaSuccess)
      return fail("survivors", e);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail("walk bound", e);
    if (o.prune_policy == 0 && hstat[0] * 4ull > walks) {
      cudaEventElapsedTime(&ms_b, r->ev0, r->ev1);
      ps.walks_kept = hstat[0];
      ps.bound_ms = ms_b;
      return plain();
    }
    if ((e = cudaLaunchKernel(ks, dim3((unsigned)blocks_s), dim3(ld::kPruneThreads), params, smem_s, s)) != cudaSuccess)
      return fail("scan launch", e);
    if ((e = cudaEventRecord(r->ev2, s)) != cudaSuccess) return fail("event", e);
  }
  if ((e = cudaMemcpyAsync(out_h, dmem + 16, sizeof(ld::Slot), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return fail("result", e);
  if ((e = cudaMemcpyAsync(hstat, dmem + off_cnt, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return fail("stats", e);
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail("solve", e);
  cudaEventElapsedTime(&ms_b, r->ev0, r->ev1);
  cudaEventElapsedTime(&ms_s, r->ev1, r->ev2);
  const ld::Slot out = *out_h;
  if (ps.incumbent != LLONG_MIN && out.value < ps.incumbent)
    return ld_fail(LD_ERR_CUDA, "internal: pruned result %lld below the incumbent %lld", (long long)out.value,
                   (long long)ps.incumbent);
  memset(res, 0, sizeof *res);
  res->value = out.value;
  res->gray_index = out.index;
  res->labelings = ld_labelings(R, d);
  res->kernel_ms = ms_b + ms_s;
  res->kernel_kind = LD_KERNEL_TABLE;
  res->lane_bits = ch.lane_bits;
  res->h2d_bytes = upload;
  res->d2h_bytes = sizeof out + 4 * sizeof(unsigned long long);
  res->evaluated = hstat[2] * (unsigned long long)B;   // high indices whose block was scanned
  if (strategy) ld_gray_labels(out.index, R, d, strategy);
  ps.pruned = 1;
  ps.walks_kept = hstat[1];
  ps.highs_kept = hstat[2];
  ps.highs_visited = hstat[3];
  ps.bound_ms = ms_b;
  ps.scan_ms = ms_s;
  if (stats) *stats = ps;
  return LD_OK;
}

// ---------------------------------------------------------------------------
// Batched solves: one persistent kernel per lane class pulling (matrix, walk
// range) chunks from a device queue (batch_kernel.cuh); the class kernels
// run concurrently on forked streams; everything is captured once into a
// CUDA graph that each ld_batch_launch replays.  Matrices outside the batch
// lane classes (d >= 4, more columns, 64-bit sums) get their own plans,
// launched inside the same graph.
#include <map>
#include <tuple>

#include "../kernels/batch_kernel.cuh"

namespace {

struct BatchClass {
  int D = 0, WB = 0, WA = 0;
  const void* kfn = nullptr;
  size_t smem = 0;
  int bps = 1;
  std::vector<int> probs;         // problem indices, largest first
  int wpt = 1;                    // walks per thread per chunk
  double grid_frac = 1.0;         // persistent CTAs per SM, as a fraction of the occupancy limit
  const void* kfn_split = nullptr;  // column-split instance (wide int32 classes), or null
  size_t smem_split = 0;
  int bps_split = 0;
  bool split = false;             // the autotuner chose the column-split instance
  float tuned[2] = {0.f, 0.f};    // autotuner: best ms per 1e9 labelings, plain / split instance
  const void* fn() const { return split ? kfn_split : kfn; }
  size_t shm() const { return split ? smem_split : smem; }
  int blocks_per_sm() const { return split ? bps_split : bps; }
  int chunk_first = 0, nchunks = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
};

// autotuner cache: (D, WB, WA, log2 of the mean walks per problem, batch_split option)
//   -> (wpt, grid fraction, split)
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int>, std::tuple<int, double, bool>> g_tune;

}  // namespace

struct ld_batch {
  int n = 0, device = 0;
  std::vector<int> R, C, d, marginal;
  std::vector<unsigned long long> labelings;
  std::vector<unsigned long long> evaluated;  // labelings the kernels compute a value for
  std::vector<int> cls;                       // class index, or -1 (own plan), or -2 (nothing to do)
  std::vector<ld_plan*> plans;                // per problem, or null
  std::vector<BatchClass> classes;
  std::vector<ld::BatchProblem> hprob;        // device pointers filled after allocation
  std::vector<ld::BatchChunk> hchunks;
  std::vector<int> range_first, range_end;
  char* dmem = nullptr;
  size_t off_prob = 0, off_chunks = 0, off_heads = 0, off_cres = 0, off_ranges = 0, off_res = 0;
  ld::Slot* hres = nullptr;                   // pinned
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool launched = false;
  std::string desc;
};

static void batch_free(ld_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto* p : b->plans) if (p) plan_free(p);
  for (auto& c : b->classes) {
    if (c.stream) cudaStreamDestroy(c.stream);
    if (c.done) cudaEventDestroy(c.done);
  }
  if (b->dmem) cudaFree(b->dmem);
  if (b->hres) cudaFreeHost(b->hres);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

// chunks of one class for a given walks-per-thread; returns the number of chunks
static int batch_chunks(const ld_batch* b, const BatchClass& c, int wpt,
                        const std::vector<unsigned long long>& walks, std::vector<ld::BatchChunk>* out) {
  const unsigned long long span = (unsigned long long)ld::kBatchThreads * (unsigned long long)wpt;
  int n = 0;
  for (int p : c.probs) {
    for (unsigned long long w = 0; w < walks[p]; w += span) {
      ld::BatchChunk ch;
      ch.walk_begin = w;
      ch.walk_end = std::min(walks[p], w + span);
      ch.problem = p;
      ch.pad = 0;
      if (out) out->push_back(ch);
      ++n;
    }
  }
  (void)b;
  return n;
}

extern "C" ld_status ld_batch_create(int32_t count, const int64_t* const* mats, const int32_t* rows,
                                     const int32_t* cols, const int32_t* ds, const int32_t* margs,
                                     const ld_options* opt, int32_t autotune, ld_batch** out) {
  if (!out || count < 1 || !mats || !rows || !cols || !ds) return ld_fail(LD_ERR_ARG, "bad batch arguments");
  ld_options o;
  if (opt) o = *opt; else ld_options_init(&o);
  DeviceInfo di;
  ld_status st = device_info(o.device, &di);
  if (st != LD_OK) return st;
  if (cudaSetDevice(o.device) != cudaSuccess) return ld_fail(LD_ERR_NODEV, "cudaSetDevice failed");
  ld_batch* b = new ld_batch();
  b->n = count;
  b->device = o.device;
  b->cls.assign(count, -2);
  b->evaluated.assign(count, 0);
  b->plans.assign(count, nullptr);
  b->range_first.assign(count, 0);
  b->range_end.assign(count, 0);
  std::vector<unsigned long long> walks(count, 0);
  std::vector<std::vector<char>> images(count);
  std::map<std::tuple<int, int, int>, int> class_of;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess) {
    batch_free(b);
    return ld_fail(LD_ERR_CUDA, "stream/event creation failed");
  }
  for (int p = 0; p < count; ++p) {
    const int R = rows[p], C = cols[p], d = ds[p], marg = margs ? margs[p] : 0;
    const int64_t* a = mats[p];
    b->R.push_back(R); b->C.push_back(C); b->d.push_back(d); b->marginal.push_back(marg);
    if (!a || R < 1 || C < 1 || d < 1 || d > LD_MAX_D || (marg && d != 1) || C > LD_MAX_COLS ||
        R > ld_max_rows_for(d) || ld_labelings(R, d) >= (1ull << 63)) {
      batch_free(b);
      return ld_fail(LD_ERR_ARG, "batch entry %d: invalid or too large (%d x %d, d=%d)", p, R, C, d);
    }
    b->labelings.push_back(ld_labelings(R, d));
    const Bounds bnd = compute_bounds(a, R, C, marg);
    const bool fits32 = !bnd.overflow && bnd.total + (marg ? bnd.K : 0) <= (long long)INT32_MAX &&
                        std::max(bnd.colbound, marg ? 2 * bnd.K : 0LL) <= (long long)INT32_MAX;
    // batch lane class: all columns int8 (WA a multiple of 4) or all int32 (WB a multiple of 8)
    Choice ch;
    int k = -1;
    const int base = d <= 2 ? 2 : d, F = R - 1;
    if (d <= 3 && fits32 && R >= 2) {
      for (int kk = std::min(F, 10); kk >= 0; --kk) {
        const unsigned long long B = ipow(base, kk);
        if (B > 1024) continue;
        Choice c;
        if (!table_config(a, R, C, d, marg, kk, 0, &c)) continue;
        c.order.clear();
        for (int l = 0; l < C; ++l) c.order.push_back(l);
        if (c.WB == 0) { c.WA = round4(c.WA); }
        else {
          c.WB = (C + 7) & ~7; c.WA = 0;
          if (c.WB > 64) continue;
          // with all-int32 lanes the column order is the identity and every column is wide
        }
        c.WT = round4(c.WB + c.WA);
        if (!ld::batch_kernel_ptr(d, c.WB, c.WA) || B * (unsigned long long)(d * c.WT) > 4096ull) continue;
        if (c.WB > 0) {      // re-pack every column as int32 (table_config may have put some in int8)
          c.order.clear();
          for (int l = 0; l < C; ++l) c.order.push_back(l);
        } else {
          // all narrow: table_config's order is identity-compatible
        }
        c.lane_bits = c.WB > 0 ? 32 : 8;
        ch = c; k = kk;
        break;
      }
    }
    if (k < 0) {                       // own plan, captured in the same graph
      ld_options po = o;
      po.stream = b->stream;
      po.shard_count = 1; po.shard_index = 0;
      ld_plan* plan = nullptr;
      st = plan_build(a, R, C, d, marg, &po, nullptr, &plan);
      if (st != LD_OK) { batch_free(b); return st; }
      b->plans[p] = plan;
      b->cls[p] = -1;
      b->evaluated[p] = plan_evaluated(plan);
      continue;
    }
    const auto key = std::make_tuple(d, ch.WB, ch.WA);
    auto it = class_of.find(key);
    int ci;
    if (it == class_of.end()) {
      ci = (int)b->classes.size();
      class_of[key] = ci;
      BatchClass bc;
      bc.D = d; bc.WB = ch.WB; bc.WA = ch.WA;
      bc.kfn = ld::batch_kernel_ptr(d, ch.WB, ch.WA);
      if (ch.WA == 0 && o.batch_split >= 0) bc.kfn_split = ld::batch_split_kernel_ptr(d, ch.WB);
      b->classes.push_back(bc);
    } else {
      ci = it->second;
    }
    b->cls[p] = ci;
    BatchClass& bc = b->classes[ci];
    bc.probs.push_back(p);
    const int nh = F - k;
    // walks per matrix: at most 2^16 (enough chunks to spread one large matrix)
    int fw = 0;
    while (fw < nh && (double)(nh - fw) * std::log2((double)base) > 16.0) ++fw;
    walks[p] = ipow(base, nh - fw);
    const int B = (int)ipow(base, k), WT = ch.WT;
    bc.smem = std::max(bc.smem, (size_t)ld::table_smem_words(d, WT, R, B) * 4);
    if (bc.kfn_split)
      bc.smem_split = std::max(bc.smem_split, (size_t)ld::batch_split_smem_words(d, ch.WB, R, B) * 4);
    // image: tot | h0 | tb | rows (each vector padded to 256 bytes)
    std::vector<int64_t> tot(C, 0), h0(C, 0), tb(C, 0);
    long long kl = 0, kh = 0;
    for (int i = 0; i < R; ++i)
      for (int l = 0; l < C; ++l) tot[l] += a[(size_t)i * C + l];
    if (d == 1) {
      for (int l = 0; l < C; ++l) h0[l] = a[(size_t)(R - 1) * C + l];
      if (marg) {
        for (int i = 0; i < R; ++i) { const int64_t v = a[(size_t)i * C]; (i < k ? kl : kh) += v < 0 ? -v : v; }
        h0[0] += kh; tb[0] = -kl;
      }
    }
    std::vector<char>& img = images[p];
    img.assign(768 + align256((size_t)R * WT * 4), 0);
    pack_row(tot.data(), ch, (uint32_t*)(img.data() + 0));
    pack_row(h0.data(), ch, (uint32_t*)(img.data() + 256));
    pack_row(tb.data(), ch, (uint32_t*)(img.data() + 512));
    for (int i = 0; i < R; ++i) pack_row(a + (size_t)i * C, ch, (uint32_t*)(img.data() + 768) + (size_t)i * WT);
    ld::BatchProblem bp{};
    bp.R = R; bp.k = k; bp.B = B; bp.fw = fw;
    bp.walk_len = ipow(base, fw);
    bp.sym_pw = 1;
    uint64_t run = walks[p];
    if (d == 3 && !o.enumerate_all && nh - fw > 0 &&
        ld_symmetry_walks(d, nh - fw, 0, walks[p], &run) == LD_OK) {
      bp.sym_digits = nh - fw;
      bp.sym_pw = ipow(base, nh - fw - 1);
    } else {
      run = walks[p];
    }
    b->evaluated[p] = (unsigned long long)run * bp.walk_len * (unsigned long long)B;
    bp.value_offset = kh + kl;
    b->hprob.resize(count);
    b->hprob[p] = bp;
  }
  b->hprob.resize(count);
  // classes: largest matrices first, occupancy, streams
  for (auto& c : b->classes) {
    std::stable_sort(c.probs.begin(), c.probs.end(),
                     [&](int x, int y) { return b->labelings[x] > b->labelings[y]; });
    if (ld_raise_smem_limit(c.kfn, c.smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c.bps, c.kfn, ld::kBatchThreads, c.smem) != cudaSuccess ||
        c.bps < 1 || cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming) != cudaSuccess) {
      batch_free(b);
      return ld_fail(LD_ERR_CUDA, "batch class D=%d WB=%d WA=%d does not fit an SM", c.D, c.WB, c.WA);
    }
    if (c.kfn_split && (ld_raise_smem_limit(c.kfn_split, c.smem_split) != cudaSuccess ||
                        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c.bps_split, c.kfn_split, ld::kBatchThreads,
                                                                      c.smem_split) != cudaSuccess ||
                        c.bps_split < 1)) {
      cudaGetLastError();
      c.kfn_split = nullptr;
    }
  }
  // device memory: images, problem table, chunks (sized for the largest wpt
  // candidate = the fewest chunks is wpt 8; the most is wpt 1), heads,
  // chunk results, ranges, results
  size_t bytes = 0;
  std::vector<size_t> img_off(count, 0);
  for (int p = 0; p < count; ++p)
    if (b->cls[p] >= 0) { img_off[p] = bytes; bytes += align256(images[p].size()); }
  int max_chunks = 0;
  for (auto& c : b->classes) max_chunks += batch_chunks(b, c, 1, walks, nullptr);
  b->off_prob = bytes;   bytes += align256(sizeof(ld::BatchProblem) * count);
  b->off_chunks = bytes; bytes += align256(sizeof(ld::BatchChunk) * std::max(1, max_chunks));
  b->off_heads = bytes;  bytes += align256(sizeof(unsigned int) * std::max<size_t>(1, b->classes.size()));
  b->off_cres = bytes;   bytes += align256(sizeof(ld::Slot) * std::max(1, max_chunks));
  b->off_ranges = bytes; bytes += align256(sizeof(int) * 2 * (size_t)count);
  b->off_res = bytes;    bytes += align256(sizeof(ld::Slot) * count);
  if (cudaMalloc(&b->dmem, bytes) != cudaSuccess || cudaMallocHost((void**)&b->hres, sizeof(ld::Slot) * count) != cudaSuccess) {
    batch_free(b);
    return ld_fail(LD_ERR_CUDA, "batch allocation of %zu bytes failed", bytes);
  }
  std::vector<char> hostimg(b->off_prob, 0);
  for (int p = 0; p < count; ++p) {
    if (b->cls[p] < 0) continue;
    memcpy(hostimg.data() + img_off[p], images[p].data(), images[p].size());
    const char* base_ptr = b->dmem + img_off[p];
    b->hprob[p].tot = (const uint32_t*)(base_ptr + 0);
    b->hprob[p].hinit = (const uint32_t*)(base_ptr + 256);
    b->hprob[p].tbias = (const uint32_t*)(base_ptr + 512);
    b->hprob[p].A = (const uint32_t*)(base_ptr + 768);
  }
  if (cudaMemcpy(b->dmem, hostimg.data(), hostimg.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->dmem + b->off_prob, b->hprob.data(), sizeof(ld::BatchProblem) * count, cudaMemcpyHostToDevice) != cudaSuccess) {
    batch_free(b);
    return ld_fail(LD_ERR_CUDA, "batch upload failed");
  }

  auto build_queue = [&]() -> ld_status {
    b->hchunks.clear();
    for (auto& c : b->classes) {
      c.chunk_first = (int)b->hchunks.size();
      c.nchunks = batch_chunks(b, c, c.wpt, walks, &b->hchunks);
    }
    for (int p = 0; p < count; ++p) { b->range_first[p] = 0; b->range_end[p] = 0; }
    for (size_t i = 0; i < b->hchunks.size(); ++i) {
      const int p = b->hchunks[i].problem;
      if (b->range_end[p] == 0) b->range_first[p] = (int)i;
      b->range_end[p] = (int)i + 1;
    }
    std::vector<int> ranges(2 * (size_t)count);
    for (int p = 0; p < count; ++p) { ranges[2 * p] = b->range_first[p]; ranges[2 * p + 1] = b->range_end[p]; }
    if (!b->hchunks.empty() &&
        cudaMemcpy(b->dmem + b->off_chunks, b->hchunks.data(), sizeof(ld::BatchChunk) * b->hchunks.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return ld_fail(LD_ERR_CUDA, "chunk upload failed");
    if (cudaMemcpy(b->dmem + b->off_ranges, ranges.data(), sizeof(int) * ranges.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return ld_fail(LD_ERR_CUDA, "range upload failed");
    return LD_OK;
  };
  auto class_args = [&](const BatchClass& c) {
    ld::BatchArgs args;
    args.problems = (const ld::BatchProblem*)(b->dmem + b->off_prob);
    args.chunks = (const ld::BatchChunk*)(b->dmem + b->off_chunks) + c.chunk_first;
    args.nchunks = c.nchunks;
    args.head = (unsigned int*)(b->dmem + b->off_heads) + (&c - b->classes.data());
    args.chunk_results = (ld::Slot*)(b->dmem + b->off_cres) + c.chunk_first;
    return args;
  };
  auto class_grid = [&](const BatchClass& c) {
    const int g = (int)std::max(1.0, std::floor((double)di.sms * c.blocks_per_sm() * c.grid_frac));
    return std::min(g, std::max(1, c.nchunks));
  };

  // autotuner: walks per thread per chunk and the persistent grid size, timed
  // on one wave of each class's chunks from its median matrix on; cached per
  // class shape and matrix size.
  for (auto& c : b->classes) {
    double mean = 0;
    for (int p : c.probs) mean += (double)walks[p];
    mean /= std::max<size_t>(1, c.probs.size());
    const auto key = std::make_tuple(c.D, c.WB, c.WA, (int)std::log2(std::max(1.0, mean)), (int)o.batch_split);
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tune.find(key);
      if (it != g_tune.end()) {
        std::tie(c.wpt, c.grid_frac, c.split) = it->second;
        if (!c.kfn_split) c.split = false;
        if (o.batch_split > 0 && c.kfn_split) c.split = true;
        continue;
      }
    }
    if (o.batch_split > 0 && c.kfn_split) c.split = true;
    if (!autotune) continue;
    float best_ms = 1e30f;
    int best_wpt = 1;
    double best_frac = 1.0;
    bool best_split = false;
    for (int variant = o.batch_split > 0 && c.kfn_split ? 1 : 0; variant < (c.kfn_split ? 2 : 1); ++variant)
    for (int wpt : {1, 2, 4, 8}) {
      for (double frac : {0.5, 1.0}) {   // persistent CTAs: half or all of the occupancy limit
        std::vector<ld::BatchChunk> all;
        batch_chunks(b, c, wpt, walks, &all);
        // one wave of chunks (a chunk per resident CTA), starting at the
        // class's median matrix: the class's steady state at a fraction of
        // the cost of its largest matrices
        const int wave = di.sms * (variant ? c.bps_split : c.bps);
        size_t first = 0;
        const int median = c.probs[c.probs.size() / 2];
        while (first < all.size() && all[first].problem != median) ++first;
        if (first + (size_t)wave > all.size()) first = all.size() > (size_t)wave ? all.size() - wave : 0;
        std::vector<ld::BatchChunk> chunks(all.begin() + first, all.end());
        const int sample = std::min<int>((int)chunks.size(), wave);
        if (sample < 1) continue;
        cudaMemcpy(b->dmem + b->off_chunks, chunks.data(), sizeof(ld::BatchChunk) * sample, cudaMemcpyHostToDevice);
        BatchClass tc = c;
        tc.chunk_first = 0; tc.nchunks = sample; tc.grid_frac = frac; tc.split = variant == 1;
        ld::BatchArgs args = class_args(c);
        args.chunks = (const ld::BatchChunk*)(b->dmem + b->off_chunks);
        args.nchunks = sample;
        args.chunk_results = (ld::Slot*)(b->dmem + b->off_cres);
        float ms = 0;
        for (int rep = 0; rep < 1; ++rep) {
          cudaMemsetAsync(args.head, 0, sizeof(unsigned int), b->stream);
          cudaEventRecord(b->ev0, b->stream);
          void* params[] = {&args};
          cudaLaunchKernel(tc.fn(), dim3(class_grid(tc)), dim3(ld::kBatchThreads), params, tc.shm(), b->stream);
          cudaEventRecord(b->ev1, b->stream);
          cudaEventSynchronize(b->ev1);
          cudaEventElapsedTime(&ms, b->ev0, b->ev1);
        }
        // normalize by the labelings the sample covered
        double lab = 0;
        for (int i = 0; i < sample; ++i)
          lab += (double)(chunks[i].walk_end - chunks[i].walk_begin) * (double)b->hprob[chunks[i].problem].walk_len *
                 (double)b->hprob[chunks[i].problem].B;
        const float per = (float)(ms / std::max(1.0, lab));
        if (per < best_ms) { best_ms = per; best_wpt = wpt; best_frac = frac; best_split = variant == 1; }
        if (c.tuned[variant] == 0.f || per * 1e9f < c.tuned[variant]) c.tuned[variant] = per * 1e9f;
      }
    }
    if (cudaGetLastError() != cudaSuccess) { batch_free(b); return ld_fail(LD_ERR_CUDA, "autotune launch failed"); }
    c.wpt = best_wpt; c.grid_frac = best_frac; c.split = best_split;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = std::make_tuple(best_wpt, best_frac, best_split);
  }
  st = build_queue();
  if (st != LD_OK) { batch_free(b); return st; }

  // capture the whole batch solve into one graph
  cudaStream_t s = b->stream;
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->dmem + b->off_heads, 0, sizeof(unsigned int) * std::max<size_t>(1, b->classes.size()), s);
  if (e == cudaSuccess) e = cudaEventRecord(b->fork, s);
  for (auto& c : b->classes) {
    if (e != cudaSuccess) break;
    e = cudaStreamWaitEvent(c.stream, b->fork, 0);
    ld::BatchArgs args = class_args(c);
    void* params[] = {&args};
    if (e == cudaSuccess && c.nchunks > 0)
      e = cudaLaunchKernel(c.fn(), dim3(class_grid(c)), dim3(ld::kBatchThreads), params, c.shm(), c.stream);
    if (e == cudaSuccess) e = cudaEventRecord(c.done, c.stream);
  }
  ld_status pst = LD_OK;
  for (int p = 0; p < count && e == cudaSuccess && pst == LD_OK; ++p)
    if (b->plans[p]) pst = plan_enqueue(b->plans[p]);
  for (auto& c : b->classes) if (e == cudaSuccess) e = cudaStreamWaitEvent(s, c.done, 0);
  if (e == cudaSuccess) {
    const ld::Slot* cres = (const ld::Slot*)(b->dmem + b->off_cres);
    const int* ranges = (const int*)(b->dmem + b->off_ranges);
    ld::Slot* res = (ld::Slot*)(b->dmem + b->off_res);
    int n = count;
    void* params[] = {(void*)&cres, (void*)&ranges, (void*)&n, (void*)&res};
    e = cudaLaunchKernel(ld::batch_fold_kernel_ptr(), dim3((count + 127) / 128), dim3(128), params, 0, s);
  }
  for (int p = 0; p < count && e == cudaSuccess; ++p)
    if (b->plans[p])
      e = cudaMemcpyAsync(b->dmem + b->off_res + sizeof(ld::Slot) * p, b->plans[p]->red.result, sizeof(ld::Slot),
                          cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b->hres, b->dmem + b->off_res, sizeof(ld::Slot) * count, cudaMemcpyDeviceToHost, s);
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(s, &g);
  if (e == cudaSuccess) e = e2;
  b->graph = g;
  if (e == cudaSuccess && pst == LD_OK) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  if (e != cudaSuccess || pst != LD_OK) {
    batch_free(b);
    return pst != LD_OK ? pst : ld_fail(LD_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(e));
  }
  char buf[256];
  snprintf(buf, sizeof buf, "%d matrices: %zu classes, %zu chunks, %d own plans", count, b->classes.size(),
           b->hchunks.size(), (int)std::count_if(b->plans.begin(), b->plans.end(), [](ld_plan* q) { return q != nullptr; }));
  b->desc = buf;
  for (auto& c : b->classes) {
    snprintf(buf, sizeof buf, "; D=%d int32=%d int8x4=%d: %zu matrices, %d chunks, wpt=%d, grid=%d%s", c.D, c.WB, c.WA,
             c.probs.size(), c.nchunks, c.wpt, class_grid(c), c.split ? ", column split" : "");
    b->desc += buf;
    if (c.tuned[0] > 0.f && c.tuned[1] > 0.f) {
      snprintf(buf, sizeof buf, " (tuned ms per 1e9 labelings: %.3f, split %.3f)", c.tuned[0], c.tuned[1]);
      b->desc += buf;
    }
  }
  *out = b;
  return LD_OK;
}

extern "C" ld_status ld_batch_launch(ld_batch* b) {
  if (!b || !b->exec) return ld_fail(LD_ERR_ARG, "null batch");
  LD_CUDA(cudaSetDevice(b->device));
  // timing events outside the graph (events recorded during capture cannot be timed)
  LD_CUDA(cudaEventRecord(b->ev0, b->stream));
  LD_CUDA(cudaGraphLaunch(b->exec, b->stream));
  LD_CUDA(cudaEventRecord(b->ev1, b->stream));
  b->launched = true;
  return LD_OK;
}

extern "C" ld_status ld_batch_results(ld_batch* b, int64_t* values, uint64_t* gray_indices, float* ms) {
  if (!b || !values) return ld_fail(LD_ERR_ARG, "null argument");
  if (!b->launched) return ld_fail(LD_ERR_ARG, "batch has not been launched");
  LD_CUDA(cudaSetDevice(b->device));
  LD_CUDA(cudaStreamSynchronize(b->stream));
  for (int p = 0; p < b->n; ++p) {
    values[p] = b->hres[p].value;
    if (gray_indices) gray_indices[p] = b->hres[p].index;
  }
  if (ms) {
    float t = 0.f;
    LD_CUDA(cudaEventElapsedTime(&t, b->ev0, b->ev1));
    *ms = t;
  }
  return LD_OK;
}

extern "C" ld_status ld_batch_describe(const ld_batch* b, char* buf, size_t cap) {
  if (!b || !buf) return ld_fail(LD_ERR_ARG, "null argument");
  snprintf(buf, cap, "%s", b->desc.c_str());
  return LD_OK;
}

extern "C" ld_status ld_batch_evaluated(const ld_batch* b, uint64_t* evaluated) {
  if (!b || !evaluated) return ld_fail(LD_ERR_ARG, "null argument");
  for (int p = 0; p < b->n; ++p) evaluated[p] = b->evaluated[p];
  return LD_OK;
}

extern "C" void ld_batch_destroy(ld_batch* b) { batch_free(b); }
