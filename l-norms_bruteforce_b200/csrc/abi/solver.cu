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
#include "solver_internal.h"
#include "../kernels/registry.h"
#include "../kernels/split_kernel.cuh"
#include "../kernels/table_kernel.cuh"
#include "../kernels/wide_kernel.cuh"
#include "device_guard.h"

using namespace ldsolve;

namespace ldsolve {



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

// Bank padding of the column-split kernel's slice regions: the S lanes of a
// group read, at step r of a tile, entry (g + r) mod S of slice g; with
// 16-byte loads a quarter warp is served in one pass when those S addresses
// fall on distinct groups of four banks.  Returns the padding (a multiple of
// 4 words, below 32) with the fewest repeated bank groups over all r.
int split_bank_pad(int S, int NW, int span) {
  int best_pad = 0, best_cost = INT_MAX;
  for (int pad = 0; pad < 32; pad += 4) {
    int cost = 0;
    for (int r = 0; r < S; ++r) {
      int cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int g = 0; g < S; ++g) cnt[((g * (span + pad) + ((g + r) % S) * NW) / 4) & 7]++;
      for (int c : cnt) cost += c > 1 ? c - 1 : 0;
    }
    if (cost < best_cost) { best_cost = cost; best_pad = pad; }
  }
  return best_pad;
}

// The column-split form of the table kernel (split_kernel.cuh), for
// matrices too wide for one thread's register vectors: over the low-row
// counts k and the (S lanes, PW words) instances whose S x PW words hold a
// row, the choice minimizing the table kernel's time estimate with the
// row padded to S x PW words, the table padded to a multiple of S entries
// and the ring's (2S - 1) instructions per labeling, divided by an
// occupancy factor: the kernel's accumulator chains and ring shuffles need
// about 16 resident warps per SM to keep the integer pipe busy, and its
// shared memory (the rows and the table in S regions) and registers decide
// how many it gets (asked from the runtime per candidate).  Lanes: all 8-bit
// when every column passes table_config's test, else all 32-bit.
static bool split_choose(const int64_t* a, int R, int C, int d, int marginal, const ld_options& o, int sms,
                         Choice* ch) {
  static const int kS[3] = {2, 4, 8};
  const int base = d <= 2 ? 2 : d, F = R - 1;
  double best_t = 0;
  bool found = false;
  for (int k = 0; k <= F; ++k) {
    const unsigned long long B = ipow(base, k);
    if (B > 1024) break;
    if (o.low_rows >= 0 && k != std::min(o.low_rows, F)) continue;
    bool narrow = o.lane_bits != 32;
    for (int l = 0; l < C && narrow; ++l) {
      long long hb = 0, lb = 0;
      for (int i = 0; i < R; ++i) {
        const int64_t v = a[(size_t)i * C + l];
        (i < k ? lb : hb) += v < 0 ? -(long long)v : (long long)v;
      }
      if (d == 1) narrow = (marginal && l == 0) ? (2 * hb <= 127 && 2 * lb <= 128) : (hb <= 127 && lb <= 127);
      else narrow = hb + lb <= 127;
    }
    if (o.lane_bits == 8 && !narrow) continue;
    const int PK = narrow ? 4 : 1;
    const int wneed = PK == 4 ? (C + 3) / 4 : C;
    double units = (double)ipow(base, F - k);
    if (d >= 3 && !o.enumerate_all && F - k > 0) {
      uint64_t pass = 0;
      if (ld_symmetry_walks(d, F - k, 0, ipow(base, F - k), &pass) == LD_OK && pass > 0) units = (double)pass;
    }
    for (int S : kS) {
      if (o.column_split > 0 && S != o.column_split) continue;
      for (int PW = 4; PW <= 32; PW += 4) {
        const void* fn = ld::table_split_kernel_ptr(d, PK, PW, S);
        if (S * PW < wneed || !fn) continue;
        const int Wp = S * PW;
        const int Bp = (int)((B + S - 1) / S * S);
        const int region = ld::split_region_words(d, PW, R, Bp);
        const size_t smem = (size_t)S * (region + 28) * sizeof(uint32_t);   // with the largest bank padding
        int bps = 0;
        if (smem > 227u * 1024u || ld_raise_smem_limit(fn, smem) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fn, ld::kTableThreads, smem) != cudaSuccess ||
            bps < 1) {
          cudaGetLastError();
          continue;
        }
        const double occ = std::min(1.0, bps * (ld::kTableThreads / 32) / 16.0);
        const double words = (double)d * Wp;
        const double per_lab = (words + (2.0 * S - 1.0) / 2.0) * (double)Bp / (double)B + (2.0 * words + 40.0) / (double)B;
        // an SM's throughput scales with the occupancy factor; groups
        // without a high index to walk add nothing
        const double groups = (double)sms * bps * (ld::kTableThreads / S);
        const double t = units * (double)B * per_lab / ((double)sms * occ) / std::min(1.0, units / groups);
        if (!found || t < best_t * 0.999) {
          best_t = t;
          found = true;
          Choice c;
          c.kind = LD_KERNEL_TABLE;
          c.D = d; c.k = k; c.S = S; c.PW = PW; c.PK = PK;
          c.WB = PK == 1 ? Wp : 0;
          c.WA = PK == 4 ? Wp : 0;
          c.WT = Wp;
          c.order.clear();
          for (int l = 0; l < C; ++l) c.order.push_back(l);
          c.lane_bits = PK == 1 ? 32 : 8;
          *ch = c;
        }
      }
    }
  }
  return found;
}

// Pick the kernel and, for the table kernel, the low-row count minimizing
// an estimate of the solve time: labelings x (words per labeling + the
// amortized cost of a high-row step) / threads that have work.
ld_status choose_kernel(const int64_t* a, int R, int C, int d, int marginal, const Bounds& b,
                        const ld_options& o, int sms, Choice* ch) {
  // threads of a full grid for the time estimate: 4 blocks of 128 per SM
  const unsigned long long full_threads = (unsigned long long)sms * 4 * 128;
  if (b.overflow) return ld_fail(LD_ERR_LIMIT, "matrix entries too large: column sums exceed 2^61");
  const long long maxabs = std::max(b.colbound, marginal ? 2 * b.K : 0LL);
  const long long vmax = b.total + (marginal ? b.K : 0LL);
  const bool fits32 = vmax <= (long long)INT32_MAX && maxabs <= (long long)INT32_MAX;
  if (o.lane_bits && o.lane_bits != 8 && o.lane_bits != 32 && o.lane_bits != 64)
    return ld_fail(LD_ERR_ARG, "lane width %d is not 8, 32 or 64", o.lane_bits);
  if (o.column_split != 0 && o.column_split != -1 && o.column_split != 2 && o.column_split != 4 &&
      o.column_split != 8)
    return ld_fail(LD_ERR_ARG, "column_split %d is not -1, 0, 2, 4 or 8", o.column_split);
  if (o.kernel != LD_KERNEL_WIDE && d <= 10 && o.lane_bits != 64 && fits32) {
    const int base = d <= 2 ? 2 : d, F = R - 1;
    double best_t = 0;
    bool found = false;
    for (int k = 0; k <= F && o.column_split <= 0; ++k) {
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
    // too wide for one thread's registers: S lanes share each high index
    if (o.column_split >= 0 && split_choose(a, R, C, d, marginal, o, sms, ch)) return LD_OK;
    if (o.column_split > 0)
      return ld_fail(LD_ERR_ARG, "no column-split instance with %d lanes takes d=%d, %d columns", o.column_split, d, C);
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

}  // namespace ldsolve

// ---------------------------------------------------------------------------
// Device resources (solver_internal.h): repeated ld_solve_reduced calls
// allocate nothing after the first.
namespace ldsolve {


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
std::mutex g_pws_mu[64];
Resources g_pws[64];




}  // namespace ldsolve


void ldsolve::plan_free(ld_plan* p) {
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
void ldsolve::split_range(unsigned long long n, int idx, int count, unsigned long long* lo,
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
ld_status ldsolve::plan_build(const int64_t* a, int R, int C, int d, int marginal, const ld_options* opt,
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
  st = choose_kernel(a, R, C, d, marginal, p->bounds, o, di.sms, &p->ch);
  if (st != LD_OK) { delete p; return st; }

  const int base = d <= 2 ? 2 : d;
  const int F = R - 1;
  std::vector<char> image;
  if (p->ch.kind == LD_KERNEL_TABLE) {
    const int D = p->ch.D, WT = p->ch.WT;
    const int S = p->ch.S > 0 ? p->ch.S : 1;   // lanes per high index (column split)
    const int k = p->ch.k;
    p->k = k;
    p->B = (int)ipow(base, k);
    p->tpb = ld::kTableThreads;
    if (p->ch.S > 0) {
      p->kfn = ld::table_split_kernel_ptr(D, p->ch.PK, p->ch.PW, p->ch.S);
      if (!p->kfn) { delete p; return ld_fail(LD_ERR_ARG, "no column-split kernel for D=%d PW=%d S=%d", D, p->ch.PW, S); }
      p->Bp = (p->B + S - 1) / S * S;
      const int region = ld::split_region_words(D, p->ch.PW, R, p->Bp);
      p->span = region + split_bank_pad(S, D * p->ch.PW, region);
      p->smem = (size_t)S * p->span * sizeof(uint32_t);
    } else {
      p->kfn = ld::table_kernel_mixed_ptr(D, p->ch.WB, p->ch.WA);
      if (!p->kfn) { delete p; return ld_fail(LD_ERR_ARG, "no table kernel for D=%d WB=%d WA=%d", D, p->ch.WB, p->ch.WA); }
      // LM with the marginal column in a 32-bit word of its own: its term is
      // never negative, so the instance that adds it linearly applies
      if (D == 1 && marginal && p->ch.WB >= 1 && !p->ch.order.empty() && p->ch.order[0] == 0) {
        if (const void* lk = ld::table_kernel_lin_ptr(p->ch.WB, p->ch.WA)) { p->kfn = lk; p->ch.lin = 1; }
      }
      p->smem = (size_t)ld::table_smem_words(D, WT, R, p->B) * sizeof(uint32_t);
    }
    if (ld_raise_smem_limit(p->kfn, p->smem) != cudaSuccess) {
      delete p; return ld_fail(LD_ERR_CUDA, "cannot reserve %zu bytes of shared memory", p->smem);
    }
    int bps = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, p->kfn, p->tpb, p->smem) != cudaSuccess || bps < 1) {
      delete p; return ld_fail(LD_ERR_CUDA, "table kernel does not fit an SM (smem %zu)", p->smem);
    }
    // packed maxima: the table kernel's scans (the column split keeps one maximum per word)
    p->pack16 = (p->ch.S == 0 && o.pack16 >= 0 && p->bounds.total + 2 * (marginal ? p->bounds.K : 0) < 65536) ? 1 : 0;
    // parallel units of a full grid: threads, or groups of S lanes
    const unsigned long long full = (unsigned long long)di.sms * bps * (p->tpb / S);
    const int nh = F - k;
    // d >= 3: walks that hold no smallest index of a label-permutation
    // class are skipped (symmetry.c); the walks that run decide the length
    const bool sym = D >= 3 && !o.enumerate_all;
    auto walks_run = [&](int f, unsigned long long lo, unsigned long long hi) -> unsigned long long {
      uint64_t c = hi - lo;
      if (sym && nh - f > 0 && ld_symmetry_walks(d, nh - f, lo, hi, &c) != LD_OK) c = hi - lo;
      return (unsigned long long)c;
    };
    // walk length: as long as the walks still number >= 16 per thread of a
    // full grid (d <= 2), or >= 4 (d >= 3, whose walk seeding costs 64-bit
    // divisions per high digit).  Longer walks seed less often; the kernel is
    // issue-bound, so warps left with one walk more than others finish
    // faster as the rest drain.  Measured: 20x30 d = 3 9 % faster at 4 than
    // at 32; 34x37 LM 3 % faster at 16 than at 32, 12 % slower at 8.
    const unsigned long long per_thread = D >= 3 ? 4ull : 16ull;
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
    const unsigned long long per_block = (unsigned long long)(p->tpb / S);
    const unsigned long long want = (mine + per_block - 1) / per_block;
    p->blocks = (int)std::min<unsigned long long>((unsigned long long)di.sms * bps, std::max(1ull, want));
    if (o.blocks > 0) p->blocks = o.blocks;
    // at least two walks per thread: the instance that walks two high
    // indices per thread against each table entry read (L_1 / LM, <= 10
    // words; d = 2, 3, <= 8 words per vector)
    if (D <= 3 && p->ch.S == 0 && o.paired_walks >= 0 &&
        mine >= 2ull * (unsigned long long)p->blocks * (unsigned long long)p->tpb) {
      const void* pk = ld::table_kernel_pair_ptr(D, p->ch.WB, p->ch.WA, p->ch.lin);
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
    // vectors of up to 64 words sit at the fixed offsets; wider ones (column
    // split) each take a multiple of 256 bytes
    const size_t vec = std::max<size_t>(256, align256((size_t)WT * 4));
    p->off_tot = kOffTot;
    p->off_h0 = kOffTot + vec;
    p->off_tb = kOffTot + 2 * vec;
    p->off_A = kOffTot + 3 * vec;
    p->upload_bytes = p->off_A + (size_t)R * WT * 4;
    if (p->sym_digits > 0) {   // completion counts for handing out walks by rank
      p->sym_off = align256(p->upload_bytes);
      p->upload_bytes = p->sym_off + ld_sym_table_len(d, p->sym_digits) * sizeof(uint64_t);
    }
    image.assign(p->upload_bytes, 0);
    if (p->sym_digits > 0) {
      const ld_status sst = ld_sym_table(d, p->sym_digits, (uint64_t*)(image.data() + p->sym_off));
      if (sst != LD_OK) { delete p; return sst; }
    }
    pack_row(tot.data(), p->ch, (uint32_t*)(image.data() + p->off_tot));
    pack_row(h0.data(), p->ch, (uint32_t*)(image.data() + p->off_h0));
    pack_row(tb.data(), p->ch, (uint32_t*)(image.data() + p->off_tb));
    for (int i = 0; i < R; ++i)
      pack_row(a + (size_t)i * C, p->ch, (uint32_t*)(image.data() + p->off_A) + (size_t)i * WT);
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
  // the table kernel's warps fetch walks from a counter in the header (zero
  // in the upload image, reset by each launch's last block)
  p->red.work = (p->ch.kind == LD_KERNEL_TABLE && p->ch.S == 0 && o.walk_fetch >= 0)
                    ? (unsigned long long*)(base_ptr + kOffWork) : nullptr;
  memcpy(p->res->hstage, image.data(), p->upload_bytes);
  cudaError_t ce = cudaMemcpyAsync(p->res->dmem, p->res->hstage, p->upload_bytes, cudaMemcpyHostToDevice,
                                   p->res->stream);
  if (ce == cudaSuccess && !shared) ce = cudaStreamSynchronize(p->res->stream);
  if (ce != cudaSuccess) { plan_free(p); return ld_fail(LD_ERR_CUDA, "upload failed: %s", cudaGetErrorString(ce)); }
  p->uploaded = true;
  *out = p;
  return LD_OK;
}

ld_status ldsolve::plan_enqueue(ld_plan* p) {
  Resources* r = p->res;
  char* base_ptr = (char*)r->dmem;
  LD_CUDA(cudaSetDevice(p->device));
  LD_CUDA(cudaEventRecord(r->ev0, r->stream));
  if (p->ch.kind == LD_KERNEL_TABLE) {
    ld::TableArgs args;
    args.A = (const uint32_t*)(base_ptr + p->off_A);
    args.tot = (const uint32_t*)(base_ptr + p->off_tot);
    args.hinit = (const uint32_t*)(base_ptr + p->off_h0);
    args.tbias = (const uint32_t*)(base_ptr + p->off_tb);
    args.R = p->R; args.k = p->k; args.B = p->B; args.fw = p->fw;
    args.walk_len = p->walk_len; args.walk_begin = p->walk_begin; args.walk_end = p->walk_end;
    args.sym_digits = p->sym_digits;
    args.sym_table = (const unsigned long long*)(base_ptr + p->sym_off);
    args.rank_begin = p->rank_begin; args.rank_end = p->rank_end;
    args.value_offset = p->value_offset;
    // every entry value in [0, 65536): the scans keep packed maxima (an
    // entry's accumulator is at most sum |A| plus twice the LM shift)
    args.pack16 = p->pack16;
    args.red = p->red;
    if (p->ch.S > 0) {
      ld::SplitArgs sargs;
      sargs.t = args;
      sargs.W = p->ch.WT;
      sargs.Bp = p->Bp;
      sargs.span = p->span;
      void* params[] = {&sargs};
      LD_CUDA(cudaLaunchKernel(p->kfn, dim3(p->blocks), dim3(p->tpb), params, p->smem, r->stream));
    } else {
      void* params[] = {&args};
      LD_CUDA(cudaLaunchKernel(p->kfn, dim3(p->blocks), dim3(p->tpb), params, p->smem, r->stream));
    }
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
unsigned long long ldsolve::plan_evaluated(const ld_plan* p) {
  if (p->ch.kind == LD_KERNEL_TABLE) return p->walks_run * p->walk_len * (unsigned long long)p->B;
  if (p->ch.kind == LD_KERNEL_WIDE)
    return p->sym_digits > 0 ? p->walks_run * p->walk_len : p->n_end - p->n_begin;
  return 0;
}

ld_status ldsolve::plan_fetch(ld_plan* p, ld_result* res, int32_t* strategy) {
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
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
  if (!out) return ld_fail(LD_ERR_ARG, "null output");
  return plan_build(a, rows, cols, d, marginal, opt, nullptr, out);
}

extern "C" ld_status ld_plan_launch(ld_plan* plan) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
  if (!plan) return ld_fail(LD_ERR_ARG, "null plan");
  return plan_enqueue(plan);
}

extern "C" ld_status ld_plan_result(ld_plan* plan, ld_result* res, int32_t* strategy) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
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
             "sym=%d blocks=%d tpb=%d smem=%zu split=%d p16=%d fetch=%d",
             p->ch.D, p->ch.WB, p->ch.WA, p->ch.lin, p->ch.pair, p->k, p->B, p->fw,
             (unsigned long long)p->walks, (unsigned long long)p->walks_run, p->sym_digits, p->blocks, p->tpb,
             p->smem, p->ch.S, p->pack16, p->red.work ? 1 : 0);
  else
    snprintf(buf, cap, "wide PC=%d multi=%d %s blocks=%d tpb=%d sym=%d walk_len=%llu run=%llu", p->ch.PC,
             p->ch.multi, p->ch.i64 ? "int64" : "int32", p->blocks, p->tpb, p->sym_digits,
             (unsigned long long)p->walk_len, (unsigned long long)p->walks_run);
  return LD_OK;
}

extern "C" void* ld_plan_stream(const ld_plan* p) { return p && p->res ? (void*)p->res->stream : nullptr; }

extern "C" void* ld_plan_result_device(const ld_plan* p) { return p ? (void*)p->red.result : nullptr; }

extern "C" void ld_plan_destroy(ld_plan* p) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
  plan_free(p);
}

extern "C" ld_status ld_solve_reduced(const int64_t* a, int32_t rows, int32_t cols, int32_t d,
                                      int32_t marginal, const ld_options* opt, ld_result* res,
                                      int32_t* strategy) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
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

