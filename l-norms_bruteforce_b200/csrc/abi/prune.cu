// Pruned exact search (prune_kernel.cuh).  Exactly the plain enumeration's
// result; the incumbent only decides how much is skipped.
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
#include "../kernels/table_kernel.cuh"

using namespace ldsolve;

#include "../kernels/prune_kernel.cuh"
#include "device_guard.h"

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
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
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
    t.pack16 = 0;
    t.red.counter = (unsigned int*)(dmem + 0);
    t.red.gvalue = (long long*)(dmem + 8);
    t.red.result = (ld::Slot*)(dmem + 16);
    t.red.slots = (ld::Slot*)(dmem + off_slots);
    t.red.work = nullptr;
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

