// Batched solves: one persistent kernel per lane class pulling (matrix, walk
// range) chunks from a device queue (batch_kernel.cuh); the class kernels
// run concurrently on forked streams; everything is captured once into a
// CUDA graph that each ld_batch_launch replays.  Matrices outside the batch
// lane classes (d >= 4, more columns, 64-bit sums) get their own plans,
// launched inside the same graph.
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

#include <map>
#include <tuple>

#include "../kernels/batch_kernel.cuh"
#include "device_guard.h"

namespace {

// threads per CTA the autotuner tries (the kernels' launch bound is 128)
constexpr int kTpbN = 2;
constexpr int kTpbChoices[kTpbN] = {64, 128};

struct BatchClass {
  int D = 0, WB = 0, WA = 0;
  const void* kfn = nullptr;
  size_t smem = 0;
  int bps = 1;                    // resident CTAs per SM at tpb threads (plain instance)
  std::vector<int> probs;         // problem indices, largest first
  int wpt = 1;                    // walks per thread per chunk
  double grid_frac = 1.0;         // persistent CTAs per SM, as a fraction of the occupancy limit
  const void* kfn_split = nullptr;  // column-split instance (wide int32 classes), or null
  size_t smem_split = 0;
  int bps_split = 0;
  bool split = false;             // the autotuner chose the column-split instance
  int tpb = ld::kBatchThreads;    // threads per CTA (chunks hold tpb * wpt walks)
  int kshift = 0;                 // low rows below the largest table that fits, for every matrix
  int occ[2][kTpbN] = {{0, 0}, {0, 0}};  // resident CTAs per SM: [split][kTpbChoices index]
  float tuned[2] = {0.f, 0.f};    // autotuner: best ms per 1e9 labelings, plain / split instance
  const void* fn() const { return split ? kfn_split : kfn; }
  size_t shm() const { return split ? smem_split : smem; }
  int blocks_per_sm() const {
    for (int t = 0; t < kTpbN; ++t)
      if (kTpbChoices[t] == tpb) return occ[split ? 1 : 0][t];
    return 0;
  }
  int chunk_first = 0, nchunks = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
};

// autotuner cache: (D, WB, WA, log2 of the mean walks per problem, batch_split option)
//   -> (wpt, grid fraction, split, threads per CTA, low-row shift)
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int>, std::tuple<int, double, bool, int, int>> g_tune;

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
  const unsigned long long span = (unsigned long long)c.tpb * (unsigned long long)wpt;
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
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
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
  std::vector<unsigned long long> max_walks(count, 0);   // over the low-row counts the tuner tries
  std::vector<std::vector<char>> images(count);
  std::vector<Choice> pch(count);                        // lane layout per class matrix
  std::vector<int> kmax(count, -1);                      // the largest low-row count that fits
  std::map<std::tuple<int, int, int>, int> class_of;
  b->hprob.resize(count);
  // walks of matrix p at low-row count k: whole high indices, at most about
  // 2^16 walks (enough chunks to spread one large matrix); fw = walked digits
  auto walk_geometry = [&](int p, int k, int* fw_out) -> unsigned long long {
    const int d = ds[p], base = d <= 2 ? 2 : d, nh = rows[p] - 1 - k;
    int fw = 0;
    while (fw < nh && (double)(nh - fw) * std::log2((double)base) > 16.0) ++fw;
    if (fw_out) *fw_out = fw;
    return ipow(base, nh - fw);
  };
  // Geometry, image and problem-table entry of class matrix p at low-row
  // count k (the device pointers of its entry are kept).  The rows' image
  // does not depend on k; for LM the initial H and the table bias do (the
  // low rows' and the other rows' share of the column-0 shift).
  auto geometry = [&](int p, int k) {
    const int R = rows[p], C = cols[p], d = ds[p], marg = margs ? margs[p] : 0;
    const int64_t* a = mats[p];
    const Choice& ch = pch[p];
    const int base = d <= 2 ? 2 : d, nh = R - 1 - k;
    int fw = 0;
    walks[p] = walk_geometry(p, k, &fw);
    const int B = (int)ipow(base, k), WT = ch.WT;
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
    ld::BatchProblem bp = b->hprob[p];   // keeps the device pointers
    bp.R = R; bp.k = k; bp.B = B; bp.fw = fw;
    bp.walk_len = ipow(base, fw);
    bp.sym_digits = 0;
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
    b->hprob[p] = bp;
  };
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
    b->classes[ci].probs.push_back(p);
    pch[p] = ch;
    kmax[p] = k;
    geometry(p, k);
    // the tuner may lower k by up to 2 for int32 classes: more walks
    max_walks[p] = ch.WA == 0 ? walk_geometry(p, std::max(0, k - 2), nullptr) : walks[p];
  }
  // a class's shared memory (its largest matrix table) and occupancy, for
  // the current geometry of its matrices
  auto class_fit = [&](BatchClass& c) -> bool {
    c.smem = 0;
    c.smem_split = 0;
    for (int p : c.probs) {
      const ld::BatchProblem& bp = b->hprob[p];
      c.smem = std::max(c.smem, (size_t)ld::table_smem_words(c.D, pch[p].WT, bp.R, bp.B) * 4);
      if (c.kfn_split)
        c.smem_split = std::max(c.smem_split, (size_t)ld::batch_split_smem_words(c.D, c.WB, bp.R, bp.B) * 4);
    }
    bool ok = ld_raise_smem_limit(c.kfn, c.smem) == cudaSuccess;
    for (int t = 0; t < kTpbN && ok; ++t)
      ok = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c.occ[0][t], c.kfn, kTpbChoices[t], c.smem) == cudaSuccess;
    c.bps = c.occ[0][1];
    if (!ok || c.bps < 1) return false;
    if (c.kfn_split) {
      bool sok = ld_raise_smem_limit(c.kfn_split, c.smem_split) == cudaSuccess;
      for (int t = 0; t < kTpbN && sok; ++t)
        sok = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c.occ[1][t], c.kfn_split, kTpbChoices[t],
                                                            c.smem_split) == cudaSuccess;
      c.bps_split = c.occ[1][1];
      if (!sok || c.bps_split < 1) {
        cudaGetLastError();
        c.kfn_split = nullptr;
      }
    }
    return true;
  };
  // classes: largest matrices first, occupancy, streams
  for (auto& c : b->classes) {
    std::stable_sort(c.probs.begin(), c.probs.end(),
                     [&](int x, int y) { return b->labelings[x] > b->labelings[y]; });
    if (!class_fit(c) || cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming) != cudaSuccess) {
      batch_free(b);
      return ld_fail(LD_ERR_CUDA, "batch class D=%d WB=%d WA=%d does not fit an SM", c.D, c.WB, c.WA);
    }
  }
  // device memory: images, problem table, chunks (sized for the largest wpt
  // candidate = the fewest chunks is wpt 8; the most is wpt 1), heads,
  // chunk results, ranges, results
  size_t bytes = 0;
  std::vector<size_t> img_off(count, 0);
  for (int p = 0; p < count; ++p)
    if (b->cls[p] >= 0) { img_off[p] = bytes; bytes += align256(images[p].size()); }
  int max_chunks = 0;   // the most chunks any candidate makes: 64 threads, 1 walk each
  for (auto& c : b->classes) {
    BatchClass tc = c;
    tc.tpb = kTpbChoices[0];
    max_chunks += batch_chunks(b, tc, 1, max_walks, nullptr);
  }
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

  // autotuner: per class, the instance (plain or column-split), threads per
  // CTA (64, 128, 256), walks per thread per chunk (1, 2, 4, 8; the chunk
  // holds threads x walks walks) and the persistent grid (half or all of the
  // occupancy limit), timed on one wave of the class's chunks from its
  // median matrix on and normalised per labeling.  Every candidate is timed
  // once; the four fastest are timed three more times and the best median
  // wins (the first launch of an instance also loads its module).  Cached
  // per class shape and matrix size.
  struct Cand { int variant, tpb, wpt; double frac; float per; };
  auto time_cand = [&](BatchClass& c, Cand& cd, int reps, float* per_out) -> ld_status {
    BatchClass tc = c;
    tc.split = cd.variant == 1;
    tc.tpb = cd.tpb;
    tc.grid_frac = cd.frac;
    const int bps = tc.blocks_per_sm();
    *per_out = 1e30f;
    if (bps < 1) return LD_OK;            // this shape does not fit an SM
    std::vector<ld::BatchChunk> all;
    batch_chunks(b, tc, cd.wpt, walks, &all);
    // one wave of chunks (a chunk per resident CTA), starting at the
    // class's median matrix: the class's steady state at a fraction of the
    // cost of its largest matrices
    const int wave = di.sms * bps;
    size_t first = 0;
    const int median = c.probs[c.probs.size() / 2];
    while (first < all.size() && all[first].problem != median) ++first;
    if (first + (size_t)wave > all.size()) first = all.size() > (size_t)wave ? all.size() - wave : 0;
    const int sample = std::min<int>((int)(all.size() - first), wave);
    if (sample < 1) return LD_OK;
    LD_CUDA(cudaMemcpy(b->dmem + b->off_chunks, all.data() + first, sizeof(ld::BatchChunk) * sample,
                       cudaMemcpyHostToDevice));
    tc.chunk_first = 0;
    tc.nchunks = sample;
    ld::BatchArgs args = class_args(c);
    args.chunks = (const ld::BatchChunk*)(b->dmem + b->off_chunks);
    args.nchunks = sample;
    args.chunk_results = (ld::Slot*)(b->dmem + b->off_cres);
    std::vector<float> ms(reps, 0.f);
    for (int rep = 0; rep < reps; ++rep) {
      LD_CUDA(cudaMemsetAsync(args.head, 0, sizeof(unsigned int), b->stream));
      LD_CUDA(cudaEventRecord(b->ev0, b->stream));
      void* params[] = {&args};
      LD_CUDA(cudaLaunchKernel(tc.fn(), dim3(class_grid(tc)), dim3(tc.tpb), params, tc.shm(), b->stream));
      LD_CUDA(cudaEventRecord(b->ev1, b->stream));
      LD_CUDA(cudaEventSynchronize(b->ev1));
      LD_CUDA(cudaEventElapsedTime(&ms[rep], b->ev0, b->ev1));
    }
    std::sort(ms.begin(), ms.end());
    // normalise by the labelings the sample covered
    double lab = 0;
    for (int i = 0; i < sample; ++i) {
      const ld::BatchChunk& q = all[first + i];
      lab += (double)(q.walk_end - q.walk_begin) * (double)b->hprob[q.problem].walk_len *
             (double)b->hprob[q.problem].B;
    }
    *per_out = (float)(ms[reps / 2] / std::max(1.0, lab));
    return LD_OK;
  };
  // the class's matrices at their largest low-row count lowered by `shift`
  // (int32 classes only: there the lane layout does not depend on k),
  // uploaded: problem-table entries and the image vectors that depend on k
  auto apply_shift = [&](BatchClass& c, int shift) -> ld_status {
    for (int p : c.probs) {
      geometry(p, std::max(0, kmax[p] - shift));
      LD_CUDA(cudaMemcpy(b->dmem + img_off[p], images[p].data(), 768, cudaMemcpyHostToDevice));
      LD_CUDA(cudaMemcpy(b->dmem + b->off_prob + sizeof(ld::BatchProblem) * p, &b->hprob[p],
                         sizeof(ld::BatchProblem), cudaMemcpyHostToDevice));
    }
    c.kshift = shift;
    if (!class_fit(c)) return ld_fail(LD_ERR_CUDA, "batch class D=%d WB=%d does not fit an SM", c.D, c.WB);
    return LD_OK;
  };
  for (auto& c : b->classes) {
    if (o.threads_per_block == 64 || o.threads_per_block == 128)
      c.tpb = o.threads_per_block;
    double mean = 0;
    for (int p : c.probs) mean += (double)walks[p];
    mean /= std::max<size_t>(1, c.probs.size());
    const auto key = std::make_tuple(c.D, c.WB, c.WA, (int)std::log2(std::max(1.0, mean)),
                                     (int)o.batch_split * 1000 + (int)o.threads_per_block * 10 +
                                         (o.batch_row_search > 0 ? 1 : 0));
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tune.find(key);
      if (it != g_tune.end()) {
        int shift = 0;
        std::tie(c.wpt, c.grid_frac, c.split, c.tpb, shift) = it->second;
        if (shift > 0) {
          st = apply_shift(c, shift);
          if (st != LD_OK) { batch_free(b); return st; }
        }
        if (!c.kfn_split) c.split = false;
        if (o.batch_split > 0 && c.kfn_split) c.split = true;
        if (c.blocks_per_sm() < 1) { c.tpb = ld::kBatchThreads; }
        continue;
      }
    }
    if (o.batch_split > 0 && c.kfn_split) c.split = true;
    if (!autotune) continue;
    // low-row counts: the largest that fits (shift 0) and, for int32
    // classes, one or two rows fewer (smaller tables, more walks)
    int max_shift = 0;
    if (c.WA == 0 && o.batch_row_search > 0)
      for (int p : c.probs) max_shift = std::max(max_shift, std::min(2, kmax[p]));
    Cand best{0, c.tpb, c.wpt, c.grid_frac, 1e30f};
    int best_shift = 0;
    for (int shift = 0; shift <= max_shift; ++shift) {
      if (shift != c.kshift) {
        st = apply_shift(c, shift);
        if (st != LD_OK) { batch_free(b); return st; }
      }
      std::vector<Cand> cands;
      for (int variant = o.batch_split > 0 && c.kfn_split ? 1 : 0; variant < (c.kfn_split ? 2 : 1); ++variant)
        for (int tpb : kTpbChoices) {
          if (o.threads_per_block > 0 && tpb != o.threads_per_block) continue;   // forced block shape
          for (int wpt : {1, 2, 4, 8})
            for (double frac : {0.5, 1.0}) cands.push_back(Cand{variant, tpb, wpt, frac, 1e30f});
        }
      for (auto& cd : cands) {
        st = time_cand(c, cd, 1, &cd.per);
        if (st != LD_OK) { batch_free(b); return st; }
      }
      std::sort(cands.begin(), cands.end(), [](const Cand& x, const Cand& y) { return x.per < y.per; });
      const size_t top = std::min<size_t>(4, cands.size());
      for (size_t i = 0; i < top; ++i) {
        st = time_cand(c, cands[i], 3, &cands[i].per);
        if (st != LD_OK) { batch_free(b); return st; }
      }
      std::sort(cands.begin(), cands.begin() + top, [](const Cand& x, const Cand& y) { return x.per < y.per; });
      for (const auto& cd : cands)
        if (c.tuned[cd.variant] == 0.f || cd.per * 1e9f < c.tuned[cd.variant]) c.tuned[cd.variant] = cd.per * 1e9f;
      if (!cands.empty() && cands[0].per < best.per) { best = cands[0]; best_shift = shift; }
    }
    if (best_shift != c.kshift) {
      st = apply_shift(c, best_shift);
      if (st != LD_OK) { batch_free(b); return st; }
    }
    if (best.per < 1e29f) {
      c.wpt = best.wpt; c.grid_frac = best.frac; c.split = best.variant == 1; c.tpb = best.tpb;
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = std::make_tuple(c.wpt, c.grid_frac, c.split, c.tpb, c.kshift);
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
      e = cudaLaunchKernel(c.fn(), dim3(class_grid(c)), dim3(c.tpb), params, c.shm(), c.stream);
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
    snprintf(buf, sizeof buf, "; D=%d int32=%d int8x4=%d: %zu matrices, %d chunks, wpt=%d, tpb=%d, k-%d, grid=%d%s",
             c.D, c.WB, c.WA, c.probs.size(), c.nchunks, c.wpt, c.tpb, c.kshift, class_grid(c),
             c.split ? ", column split" : "");
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
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
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
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
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

extern "C" void ld_batch_destroy(ld_batch* b) {
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
  batch_free(b);
}
