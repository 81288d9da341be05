/*
 * Label symmetry of L_d for d >= 3 (no counterpart in the reference, which
 * enumerates every labeling with the last row fixed: L_CUDA.cu:186-240,
 * L_OpenMP.c).
 *
 * The fixed row carries label 0, and the value sum_k sum_l |s_k,l| is
 * unchanged when labels 1..d-1 are permuted, so the labelings fall into
 * classes of equal value.  The reference reports the smallest Gray index
 * attaining the maximum; that index is the smallest of its class.
 *
 * The table kernel walks blocks of high indices whose top digits (the walk
 * prefix, P base-d digits of the walk number) are fixed.  Read from the top,
 * each label that appears for the first time at a digit could instead take
 * any label not seen above it, through a permutation that leaves the labels
 * above untouched (so the reflection of the digit is unchanged).  When an
 * unseen label would give a smaller digit there, that permutation lowers
 * every index of the walk, so the walk holds no class minimum and can be
 * skipped without changing the value or the reported index.  The test: the
 * first appearance of each label takes the smallest digit any unseen label
 * could take (the smallest unseen label where the digit is read directly,
 * the largest where it is mirrored).  Once at most one label is unseen the
 * rest of the prefix always passes.
 *
 * The device copy of the test is walk_holds_class_min in table_kernel.cuh;
 * this file counts the walks that pass (a digit DP), for the walk length,
 * the split of a solve into shards of equal work and the evaluated-labelings
 * count of a result.
 */
#include <stdlib.h>

#include "ld_internal.h"

/* reflection of the digit below one with reflection `par` and value n:
 * parity of floor(N / d^(q)) from that of floor(N / d^(q+1)) */
static int sym_next_par(int d, int par, int n) { return (d & 1) ? (par ^ (n & 1)) : (n & 1); }

/* the label an unseen label must be where it first appears */
static int sym_want(int d, unsigned used, int par) {
    const unsigned unused = ~used & ((1u << d) - 1u);
    if (!unused) return -1;
    if (par) return 31 - __builtin_clz(unused);
    return __builtin_ctz(unused);
}

static int sym_free(int d, unsigned used) { return d - __builtin_popcount(used); }

int32_t ld_symmetry_walk_ok(int32_t d, int32_t P, uint64_t w) {
    if (d < 3 || d > LD_MAX_D || P <= 0) return 1;
    uint64_t pw = 1;
    for (int q = 1; q < P; q++) pw *= (uint64_t)d;
    if (w / pw >= (uint64_t)d) return 0;   /* not a P-digit walk number */
    unsigned used = 1u;
    int par = 0;
    uint64_t rem = w;
    for (int q = P - 1; q >= 0 && sym_free(d, used) > 1; q--) {
        const int n = (int)(rem / pw);
        rem -= (uint64_t)n * pw;
        const int lab = par ? d - 1 - n : n;
        if (!((used >> lab) & 1u)) {
            if (lab != sym_want(d, used, par)) return 0;
            used |= 1u << lab;
        }
        par = sym_next_par(d, par, n);
        pw /= (uint64_t)d;
    }
    return 1;
}

typedef struct {
    int d, P;
    uint64_t *memo;   /* [used >> 1][par][r], UINT64_MAX = not computed */
} sym_ctx;

static uint64_t upow(int d, int r) {
    uint64_t t = 1;
    for (int i = 0; i < r; i++) t *= (uint64_t)d;
    return t;
}

/* passing completions of r more digits after a prefix with labels `used`
 * whose next digit has reflection par */
static uint64_t sym_completions(sym_ctx *c, unsigned used, int par, int r) {
    const int d = c->d;
    if (r == 0) return 1;
    if (sym_free(d, used) <= 1) return upow(d, r);
    uint64_t *m = &c->memo[(((size_t)(used >> 1) * 2 + (size_t)par) * (size_t)(c->P + 1)) + (size_t)r];
    if (*m != UINT64_MAX) return *m;
    const int want = sym_want(d, used, par);
    uint64_t s = 0;
    for (int n = 0; n < d; n++) {
        const int lab = par ? d - 1 - n : n;
        if (((used >> lab) & 1u) || lab == want)
            s += sym_completions(c, used | (1u << lab), sym_next_par(d, par, n), r - 1);
    }
    *m = s;
    return s;
}

static int sym_init(sym_ctx *c, int d, int P) {
    c->d = d;
    c->P = P;
    const size_t n = ((size_t)1 << (d - 1)) * 2 * (size_t)(P + 1);
    c->memo = (uint64_t *)malloc(n * sizeof(uint64_t));
    if (!c->memo) return 0;
    for (size_t i = 0; i < n; i++) c->memo[i] = UINT64_MAX;
    return 1;
}

/* passing walks w' < w (0 <= w <= d^P) */
static uint64_t sym_below(sym_ctx *c, uint64_t w) {
    const int d = c->d, P = c->P;
    uint64_t pw = upow(d, P - 1);
    if (w >= pw * (uint64_t)d) return sym_completions(c, 1u, 0, P);
    unsigned used = 1u;
    int par = 0;
    uint64_t rem = w, total = 0;
    for (int q = P - 1; q >= 0; q--) {
        if (sym_free(d, used) <= 1) return total + rem;   /* every suffix passes */
        const int nq = (int)(rem / pw);
        rem -= (uint64_t)nq * pw;
        const int want = sym_want(d, used, par);
        for (int n = 0; n < nq; n++) {
            const int lab = par ? d - 1 - n : n;
            if (((used >> lab) & 1u) || lab == want)
                total += sym_completions(c, used | (1u << lab), sym_next_par(d, par, n), q);
        }
        const int lab = par ? d - 1 - nq : nq;
        if (!((used >> lab) & 1u)) {
            if (lab != want) return total;   /* no walk with this prefix passes */
            used |= 1u << lab;
        }
        par = sym_next_par(d, par, nq);
        pw /= (uint64_t)d;
    }
    return total;
}

ld_status ld_symmetry_walks(int32_t d, int32_t P, uint64_t lo, uint64_t hi, uint64_t *count) {
    if (!count || lo > hi) return ld_fail(LD_ERR_ARG, "bad walk range");
    if (d < 3 || P <= 0) { *count = hi - lo; return LD_OK; }
    if (d > LD_MAX_D || (double)P * __builtin_log2((double)d) >= 63.0)
        return ld_fail(LD_ERR_ARG, "prefix of %d base-%d digits", P, d);
    const uint64_t W = upow(d, P);
    if (hi > W) return ld_fail(LD_ERR_ARG, "walk range beyond %llu", (unsigned long long)W);
    sym_ctx c;
    if (!sym_init(&c, d, P)) return ld_fail(LD_ERR_NOMEM, "symmetry table");
    *count = sym_below(&c, hi) - sym_below(&c, lo);
    free(c.memo);
    return LD_OK;
}

size_t ld_sym_table_len(int d, int P) { return ((size_t)1 << (d - 1)) * 2 * (size_t)(P + 1); }

ld_status ld_sym_table(int d, int P, uint64_t *table) {
    if (d < 3 || d > LD_MAX_D || P <= 0) return ld_fail(LD_ERR_ARG, "no symmetry table for d=%d, %d digits", d, P);
    sym_ctx c;
    if (!sym_init(&c, d, P)) return ld_fail(LD_ERR_NOMEM, "symmetry table");
    for (unsigned u = 1; u < (1u << d); u += 2)
        for (int par = 0; par < 2; par++)
            for (int r = 0; r <= P; r++)
                table[(((size_t)(u >> 1) * 2 + (size_t)par) * (size_t)(P + 1)) + (size_t)r] =
                    sym_completions(&c, u, par, r);
    free(c.memo);
    return LD_OK;
}

/* The passing walk of a given rank (0-based, increasing walk numbers), from
 * the completion counts f[(used >> 1)][par][r] of ld_sym_table.  The device
 * copy is walk_of_rank in table_kernel.cuh. */
static uint64_t sym_walk_of_rank(int d, int P, const uint64_t *f, uint64_t i) {
    unsigned used = 1u;
    int par = 0, q = P - 1;
    uint64_t w = 0;
    for (; q >= 0 && sym_free(d, used) > 1; q--) {
        const int want = sym_want(d, used, par);
        int n = 0, lab = 0, np = 0;
        for (n = 0; n < d; n++) {
            lab = par ? d - 1 - n : n;
            if (!(((used >> lab) & 1u) || lab == want)) continue;
            np = sym_next_par(d, par, n);
            const uint64_t c = f[(((size_t)((used | (1u << lab)) >> 1) * 2 + (size_t)np) * (size_t)(P + 1)) + (size_t)q];
            if (i < c) break;
            i -= c;
        }
        if (n == d) return UINT64_MAX;   /* rank beyond the passing walks */
        w = w * (uint64_t)d + (uint64_t)n;
        used |= 1u << lab;
        par = np;
    }
    /* every suffix of the remaining q + 1 digits passes: in numeric order */
    for (int t = 0; t <= q; t++) w *= (uint64_t)d;
    return w + i;
}

ld_status ld_symmetry_walk_at(int32_t d, int32_t P, uint64_t rank, uint64_t *w) {
    if (!w) return ld_fail(LD_ERR_ARG, "null output");
    if (d < 3 || P <= 0) { *w = rank; return LD_OK; }
    if (d > LD_MAX_D || (double)P * __builtin_log2((double)d) >= 63.0)
        return ld_fail(LD_ERR_ARG, "prefix of %d base-%d digits", P, d);
    uint64_t *f = (uint64_t *)malloc(ld_sym_table_len(d, P) * sizeof(uint64_t));
    if (!f) return ld_fail(LD_ERR_NOMEM, "symmetry table");
    ld_status st = ld_sym_table(d, P, f);
    if (st == LD_OK) {
        const uint64_t K = f[(size_t)0 * (size_t)(P + 1) + (size_t)P];   /* used = {0}, par 0, P digits */
        if (rank >= K) st = ld_fail(LD_ERR_ARG, "rank %llu of %llu passing walks", (unsigned long long)rank,
                                    (unsigned long long)K);
        else *w = sym_walk_of_rank(d, P, f, rank);
    }
    free(f);
    return st;
}

ld_status ld_sym_split(int d, int P, int index, int count, uint64_t *lo, uint64_t *hi) {
    if (!lo || !hi || count < 1 || index < 0 || index >= count) return ld_fail(LD_ERR_ARG, "bad shard");
    if (d > LD_MAX_D || (double)P * __builtin_log2((double)(d < 2 ? 2 : d)) >= 63.0)
        return ld_fail(LD_ERR_ARG, "prefix of %d base-%d digits", P, d);
    const uint64_t W = upow(d < 3 ? 2 : d, P < 0 ? 0 : P);
    sym_ctx c;
    int sym = d >= 3 && P > 0;
    if (sym && !sym_init(&c, d, P)) return ld_fail(LD_ERR_NOMEM, "symmetry table");
    const uint64_t K = sym ? sym_below(&c, W) : W;
    uint64_t b[2];
    for (int e = 0; e < 2; e++) {
        const int s = index + e;
        if (s == 0) { b[e] = 0; continue; }
        if (s == count) { b[e] = W; continue; }
        /* the first walk w with at least K*s/count passing walks below it */
        const uint64_t target = K / (uint64_t)count * (uint64_t)s + K % (uint64_t)count * (uint64_t)s / (uint64_t)count;
        uint64_t a = 0, z = W;
        while (a < z) {
            const uint64_t mid = a + (z - a) / 2;
            if ((sym ? sym_below(&c, mid) : mid) >= target) z = mid; else a = mid + 1;
        }
        b[e] = a;
    }
    if (sym) free(c.memo);
    *lo = b[0];
    *hi = b[1];
    return LD_OK;
}
