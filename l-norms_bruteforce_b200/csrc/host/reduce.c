/*
 * Preprocessing: the reduction rules of load_parameters (L_CUDA.cu:414-423)
 * with the same observable behaviour (stdout lines, reduced matrix, line
 * bookkeeping for the strategy file).
 *
 *  1. zero lines (flags y/r/c): eliminate_zero_rows_cols, functions.h:109-151
 *  2. row uniting (flags y/r): calc_reduce_matrix_rows, functions.h:237-262
 *  3. column uniting (flags y/c): calc_reduce_matrix_cols, :264-289, then for
 *     d > 1 the same-sign column merge calc_reduce_matrix_cols_sign, :193-235
 *  4. compaction, flattening, transpose for d == 1 with rows > cols, and the
 *     marginal row swap: delete_rows/cols + convert_mtx_to_vec, :153-191, :291-329
 *  5. the d reset of calc_Parameters (L_CUDA.cu:244-248)
 *
 * Uniting is done here by grouping lines on a canonical direction (the line
 * divided by the gcd of its entries, oriented so its first nonzero entry is
 * positive) instead of the reference's pairwise cross-product scan.  Two
 * integer lines are proportional exactly when their canonical directions
 * agree, so the groups are the reference's; each group's smallest index
 * absorbs the others in increasing order, which reproduces its messages and
 * their order.  Adding a proportional line only rescales the absorbing line
 * by a positive factor, so grouping on the input lines equals the
 * reference's tests on the progressively modified matrix.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ld_internal.h"

static int prep_any(char c) { return strchr("yYrRcC", c) != NULL && c != 0; }
static int prep_rows(char c) { return c == 'y' || c == 'Y' || c == 'r' || c == 'R'; }
static int prep_cols(char c) { return c == 'y' || c == 'Y' || c == 'c' || c == 'C'; }

#define AT(p, i, j) ((p)->a[(size_t)(i) * (p)->C0 + (j)])

int ld_max_rows_for(int d) {
    if (d <= 2) return LD_INDEX_BITS - 1;
    return (int)(floor(LD_INDEX_BITS / log2((double)d)) + 1);
}

uint64_t ld_labelings(int rows, int d) {
    if (rows <= 0) return 0;
    uint64_t base = d <= 2 ? 2 : (uint64_t)d, t = 1;
    for (int i = 0; i < rows - 1; i++) {
        if (t > UINT64_MAX / base) return UINT64_MAX;
        t *= base;
    }
    return t;
}

/* ---- canonical directions ------------------------------------------- */
typedef struct {
    const int64_t *canon;   /* n entries per line                 */
    const int *orient;      /* +1 / -1: sign of the first nonzero */
    int n;
    int signed_key;         /* group parallel lines only          */
} canon_ctx;

static uint64_t gcd_u64(uint64_t a, uint64_t b) {
    while (b) { uint64_t t = a % b; a = b; b = t; }
    return a;
}

/* line x (n entries, stride s) -> canonical direction c and orientation */
static void canonical(const int64_t *x, int n, size_t s, int64_t *c, int *orient) {
    uint64_t g = 0; int first = -1;
    for (int k = 0; k < n; k++) {
        int64_t v = x[k * s];
        if (v != 0) {
            if (first < 0) first = k;
            uint64_t av = v < 0 ? (uint64_t)0 - (uint64_t)v : (uint64_t)v;
            g = gcd_u64(g, av);
        }
    }
    int o = (first >= 0 && x[first * s] < 0) ? -1 : 1;
    for (int k = 0; k < n; k++) {
        int64_t v = x[k * s];
        c[k] = g ? (int64_t)(o * (v / (int64_t)g)) : 0;
    }
    *orient = o;
}

static int cmp_lines(const void *pa, const void *pb, void *pc) {
    const canon_ctx *cx = (const canon_ctx *)pc;
    int ia = *(const int *)pa, ib = *(const int *)pb;
    const int64_t *ca = cx->canon + (size_t)ia * cx->n, *cb = cx->canon + (size_t)ib * cx->n;
    for (int k = 0; k < cx->n; k++)
        if (ca[k] != cb[k]) return ca[k] < cb[k] ? -1 : 1;
    if (cx->signed_key && cx->orient[ia] != cx->orient[ib]) return cx->orient[ia] < cx->orient[ib] ? -1 : 1;
    return ia < ib ? -1 : (ia > ib);
}

typedef struct { int leader, member, sign; } merge_t;

static int cmp_merge(const void *pa, const void *pb) {
    const merge_t *a = (const merge_t *)pa, *b = (const merge_t *)pb;
    if (a->leader != b->leader) return a->leader < b->leader ? -1 : 1;
    return a->member < b->member ? -1 : (a->member > b->member);
}

/* Unite proportional lines.  rows != 0: lines are rows, else columns.
 * keep_anti: unite anti-parallel lines too (columns always; rows for d==1). */
static ld_status unite(ld_problem *p, int rows, int keep_anti) {
    int nl = rows ? p->R0 : p->C0;       /* number of lines      */
    int len = rows ? p->C0 : p->R0;      /* entries per line     */
    int *mark = rows ? p->rmark : p->cmark;
    int start = p->marg_user;            /* marginal line never unites */
    int64_t *canon = (int64_t *)malloc((size_t)nl * len * sizeof(int64_t));
    int *orient = (int *)malloc((size_t)nl * sizeof(int));
    int *idx = (int *)malloc((size_t)nl * sizeof(int));
    merge_t *mg = (merge_t *)malloc((size_t)nl * sizeof(merge_t));
    if (!canon || !orient || !idx || !mg) {
        free(canon); free(orient); free(idx); free(mg);
        return ld_fail(LD_ERR_NOMEM, "out of host memory in preprocessing");
    }
    int m = 0;
    for (int i = start; i < nl; i++) {
        if (mark[i] != 0) continue;
        const int64_t *x = rows ? &AT(p, i, 0) : &AT(p, 0, i);
        canonical(x, len, rows ? 1 : (size_t)p->C0, canon + (size_t)i * len, &orient[i]);
        idx[m++] = i;
    }
    canon_ctx cx = {canon, orient, len, !keep_anti};
    qsort_r(idx, (size_t)m, sizeof(int), cmp_lines, &cx);
    int nm = 0;
    for (int s = 0; s < m;) {
        int e = s + 1;
        while (e < m) {
            int a = idx[s], b = idx[e];
            /* same key: compare without the index tie-break */
            const int64_t *ca = canon + (size_t)a * len, *cb = canon + (size_t)b * len;
            if (memcmp(ca, cb, (size_t)len * sizeof(int64_t)) != 0) break;
            if (!keep_anti && orient[a] != orient[b]) break;
            e++;
        }
        int leader = idx[s];   /* sorted by index inside the group */
        for (int t = s + 1; t < e; t++)
            mg[nm++] = (merge_t){leader, idx[t], orient[idx[t]] * orient[leader]};
        s = e;
    }
    qsort(mg, (size_t)nm, sizeof(merge_t), cmp_merge);
    for (int t = 0; t < nm; t++) {
        int i = mg[t].leader, j = mg[t].member, sg = mg[t].sign;
        mark[j] = sg > 0 ? i + 1 : -(i + 1);
        if (rows) {
            for (int k = 0; k < p->C0; k++) AT(p, i, k) += sg * AT(p, j, k);
            ld_logf(p, sg > 0 ? "row %d was added to %d\n" : "row %d was subtracted from %d\n", j + 1, i + 1);
        } else {
            for (int k = 0; k < p->R0; k++) AT(p, k, i) += sg * AT(p, k, j);
            ld_logf(p, sg > 0 ? "col %d was added to %d\n" : "col %d was subtracted from %d\n", j + 1, i + 1);
        }
    }
    if (rows) p->R -= nm; else p->C -= nm;
    free(canon); free(orient); free(idx); free(mg);
    return LD_OK;
}

/* eliminate_zero_rows_cols (functions.h:109-151): with marginals the first
 * row / column is kept even if zero, unless both are zero, in which case the
 * marginal treatment is switched off and both are dropped. */
static void zero_lines(ld_problem *p) {
    int cr = 0, cc = 0;
    for (int i = 0; i < p->R0; i++) {
        int z = 1;
        for (int k = 0; k < p->C0 && z; k++) z = AT(p, i, k) == 0;
        if (z) {
            p->rmark[i] = p->R0;
            if (!p->marg_user || i > 0) { cr++; ld_logf(p, "row %d entries are zeros.\n", i + 1); }
        }
    }
    p->R = p->R0 - cr;
    for (int j = 0; j < p->C0; j++) {
        int z = 1;
        for (int k = 0; k < p->R0 && z; k++) z = AT(p, k, j) == 0;
        if (z) {
            p->cmark[j] = p->C0;
            if (!p->marg_user || j > 0) { cc++; ld_logf(p, "col %d entries are zeros.\n", j + 1); }
        }
    }
    p->C = p->C0 - cc;
    if (p->marg_user) {
        if (p->rmark[0] == p->R0 && p->cmark[0] == p->C0) {
            p->marg = 0; p->R--; p->C--;
            ld_logf(p, "The entries of the first row and column are zeros.\n");
        } else {
            p->rmark[0] = 0; p->cmark[0] = 0;
        }
    }
}

/* calc_reduce_matrix_cols_sign (functions.h:193-235), d > 1 only: a column
 * whose entries all share one sign contributes the same amount to every
 * labeling, so all such columns fold into the first one. */
static void fold_single_sign_columns(ld_problem *p) {
    int *sg = (int *)calloc((size_t)p->C0, sizeof(int));
    int cnt = 0, first = -1;
    for (int j = 0; j < p->C0; j++) {
        if (p->cmark[j] != 0) continue;
        int pos = 0, neg = 0;
        for (int k = 0; k < p->R0 && !(pos && neg); k++) {
            pos |= AT(p, k, j) > 0;
            neg |= AT(p, k, j) < 0;
        }
        sg[j] = (pos && neg) ? 0 : (neg ? -1 : 1);
        if (sg[j]) { cnt++; if (first < 0) first = j; }
    }
    if (cnt > 1) {
        p->C -= cnt - 1;
        for (int j = first + 1; j < p->C0; j++) {
            if (p->cmark[j] != 0 || sg[j] == 0) continue;
            int s = sg[first] * sg[j];
            p->cmark[j] = s > 0 ? first + 1 : -(first + 1);
            for (int k = 0; k < p->R0; k++) AT(p, k, first) += s * AT(p, k, j);
            ld_logf(p, s > 0 ? "col %d was added to %d\n" : "col %d was subtracted from %d\n", j + 1, first + 1);
        }
    }
    free(sg);
}

/* delete_rows / delete_cols / convert_mtx_to_vec (functions.h:153-191, 291-329). */
static ld_status flatten(ld_problem *p) {
    int prep = prep_any(p->stat);
    int *ri = (int *)malloc(sizeof(int) * (size_t)(p->R0 + 1));
    int *ci = (int *)malloc(sizeof(int) * (size_t)(p->C0 + 1));
    size_t cells = (size_t)(p->R > 0 ? p->R : 1) * (size_t)(p->C > 0 ? p->C : 1);
    p->red = (int64_t *)calloc(cells, sizeof(int64_t));
    if (!ri || !ci || !p->red) { free(ri); free(ci); return ld_fail(LD_ERR_NOMEM, "out of host memory"); }
    int nr = 0, nc = 0;
    for (int i = 0; i < p->R0; i++) if (!prep || p->rmark[i] == 0) ri[nr++] = i;
    for (int j = 0; j < p->C0; j++) if (!prep || p->cmark[j] == 0) ci[nc++] = j;
    if (nr != p->R || nc != p->C) {
        free(ri); free(ci);
        return ld_fail(LD_ERR_INPUT, "internal: reduced counts disagree (%d/%d, %d/%d)", nr, p->R, nc, p->C);
    }
    if (p->d_user == 1 && p->R > p->C) {
        for (int j = 0; j < p->C; j++)
            for (int i = 0; i < p->R; i++) p->red[(size_t)j * p->R + i] = AT(p, ri[i], ci[j]);
        int t = p->R; p->R = p->C; p->C = t;
        p->orig = p->cmark; p->orig_len = p->C0; p->transposed = 1;
        ld_logf(p, "Matrix was transposed.\n");
    } else {
        for (int i = 0; i < p->R; i++)
            for (int j = 0; j < p->C; j++) p->red[(size_t)i * p->C + j] = AT(p, ri[i], ci[j]);
        p->orig = p->rmark; p->orig_len = p->R0; p->transposed = 0;
    }
    /* the marginal row (first kept) goes to the fixed, last position */
    if (p->marg && p->R > 1)
        for (int j = 0; j < p->C; j++) {
            int64_t t = p->red[(size_t)(p->R - 1) * p->C + j];
            p->red[(size_t)(p->R - 1) * p->C + j] = p->red[j];
            p->red[j] = t;
        }
    free(ri); free(ci);
    return LD_OK;
}

ld_status ld_problem_build(int64_t *a, int rows, int cols, int d, char stat, int marginal,
                           ld_problem **out) {
    ld_problem *p = (ld_problem *)calloc(1, sizeof(ld_problem));
    if (!p) { free(a); return ld_fail(LD_ERR_NOMEM, "out of host memory"); }
    p->R0 = rows; p->C0 = cols; p->a = a;
    p->d_user = d; p->stat = stat; p->marg_user = (d == 1 && marginal) ? 1 : 0;
    p->rmark = (int *)calloc((size_t)rows, sizeof(int));
    p->cmark = (int *)calloc((size_t)cols, sizeof(int));
    if (!p->rmark || !p->cmark) { ld_problem_destroy(p); return ld_fail(LD_ERR_NOMEM, "out of host memory"); }
    ld_logf(p, "rows: %d, cols: %d\n", rows, cols);
    p->R = rows; p->C = cols; p->marg = p->marg_user;
    ld_status st = LD_OK;
    if (prep_any(stat)) zero_lines(p);
    if (prep_rows(stat)) st = unite(p, 1, d == 1);
    if (st == LD_OK && prep_cols(stat)) {
        st = unite(p, 0, 1);
        if (st == LD_OK && d > 1) fold_single_sign_columns(p);
    }
    if (st == LD_OK) st = flatten(p);
    if (st != LD_OK) { ld_problem_destroy(p); return st; }
    /* d reset (L_CUDA.cu:244-248) */
    if (d < p->R || d == 1) p->d = d;
    else {
        p->d = p->R > 1 ? p->R : 2;
        ld_logf(p, "The preprocessed matrix has a number of rows (%d) less than or equal to the order of the L norm (%d).\n", p->R, d);
    }
    p->max_rows = ld_max_rows_for(p->d);
    p->labelings = ld_labelings(p->R, p->d);
    *out = p;
    return LD_OK;
}
