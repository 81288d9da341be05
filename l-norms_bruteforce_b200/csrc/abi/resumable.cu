// Resumable solves: the shards of one solve run one after another, with a
// checkpoint after each (no counterpart in the reference, whose runs cannot
// be interrupted and resumed).
#include <climits>
#include <cstdio>
#include <cstring>
#include <string>

#include "solver_internal.h"
#include "device_guard.h"

using namespace ldsolve;

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
  ldsolve::ContextRestore ctx_restore;   // the caller's current context, back on return
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

