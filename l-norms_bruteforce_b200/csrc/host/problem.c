/*
 * Problem objects, the launch-line / limit checks of calc_Parameters, the
 * strategy-file reconstruction of print_results, and error reporting.
 */
#define _GNU_SOURCE
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ld_internal.h"

/* ---- errors --------------------------------------------------------- */
static __thread char g_err[512];

ld_status ld_fail(ld_status st, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return st;
}

void ld_clear_error(void) { g_err[0] = 0; }
const char *ld_last_error(void) { return g_err; }
const char *ld_version(void) { return "lnorms_b200 0.1 (sm_100a)"; }

/* ---- stdout text ---------------------------------------------------- */
void ld_logf(ld_problem *p, const char *fmt, ...) {
    char tmp[1024];
    va_list ap;
    va_start(ap, fmt);
    int k = vsnprintf(tmp, sizeof tmp, fmt, ap);
    va_end(ap);
    if (k < 0) return;
    if ((size_t)k >= sizeof tmp) k = (int)sizeof tmp - 1;
    if (p->log_n + (size_t)k + 1 > p->log_cap) {
        size_t nc = (p->log_cap + (size_t)k + 1) * 2;
        char *np = (char *)realloc(p->log, nc);
        if (!np) return;
        p->log = np; p->log_cap = nc;
    }
    memcpy(p->log + p->log_n, tmp, (size_t)k);
    p->log_n += (size_t)k;
    p->log[p->log_n] = 0;
}

const char *ld_problem_log(const ld_problem *p) { return p && p->log ? p->log : ""; }

/* ---- construction --------------------------------------------------- */
ld_status ld_problem_from_text(const char *text, size_t len, int32_t d, char stat,
                               int32_t marginal, ld_problem **out) {
    if (!text || !out) return ld_fail(LD_ERR_ARG, "null argument");
    if (d < 1 || d > LD_MAX_D) return ld_fail(LD_ERR_ARG, "order d=%d outside 1..%d", d, LD_MAX_D);
    int64_t *a; int r, c;
    ld_status st = ld_parse_matrix_text(text, len, &a, &r, &c);
    if (st != LD_OK) return st;
    return ld_problem_build(a, r, c, d, stat, marginal, out);
}

ld_status ld_problem_from_file(const char *path, int32_t d, char stat, int32_t marginal,
                               ld_problem **out) {
    if (!path || !out) return ld_fail(LD_ERR_ARG, "null argument");
    FILE *f = fopen(path, "rb");
    if (!f) return ld_fail(LD_ERR_IO, "cannot open %s", path);
    size_t cap = 1 << 16, n = 0;
    char *buf = (char *)malloc(cap);
    for (;;) {
        if (!buf) { fclose(f); return ld_fail(LD_ERR_NOMEM, "out of host memory"); }
        size_t k = fread(buf + n, 1, cap - n, f);
        n += k;
        if (n < cap) break;
        cap *= 2;
        char *nb = (char *)realloc(buf, cap);
        if (!nb) free(buf);
        buf = nb;
    }
    fclose(f);
    ld_status st = ld_problem_from_text(buf, n, d, stat, marginal, out);
    free(buf);
    return st;
}

ld_status ld_problem_from_matrix(const int64_t *a, int32_t rows, int32_t cols, int32_t d,
                                 char stat, int32_t marginal, ld_problem **out) {
    if (!a || !out || rows < 1 || cols < 1) return ld_fail(LD_ERR_ARG, "bad matrix arguments");
    if (d < 1 || d > LD_MAX_D) return ld_fail(LD_ERR_ARG, "order d=%d outside 1..%d", d, LD_MAX_D);
    int64_t *copy = (int64_t *)malloc((size_t)rows * cols * sizeof(int64_t));
    if (!copy) return ld_fail(LD_ERR_NOMEM, "out of host memory");
    memcpy(copy, a, (size_t)rows * cols * sizeof(int64_t));
    return ld_problem_build(copy, rows, cols, d, stat, marginal, out);
}

void ld_problem_destroy(ld_problem *p) {
    if (!p) return;
    free(p->a); free(p->rmark); free(p->cmark); free(p->red); free(p->log);
    free(p);
}

ld_status ld_problem_get_info(const ld_problem *p, ld_problem_info *info) {
    if (!p || !info) return ld_fail(LD_ERR_ARG, "null argument");
    info->rows_in = p->R0; info->cols_in = p->C0;
    info->rows = p->R; info->cols = p->C;
    info->d_user = p->d_user; info->d = p->d;
    info->marginal_user = p->marg_user; info->marginal = p->marg;
    info->transposed = p->transposed;
    info->max_rows = p->max_rows;
    info->labelings = p->labelings;
    return LD_OK;
}

ld_status ld_problem_reduced(const ld_problem *p, int64_t *out, size_t cap) {
    if (!p || (!out && p->R > 0)) return ld_fail(LD_ERR_ARG, "null argument");
    size_t n = (size_t)p->R * p->C;
    if (cap < n) return ld_fail(LD_ERR_ARG, "buffer holds %zu entries, need %zu", cap, n);
    if (n) memcpy(out, p->red, n * sizeof(int64_t));
    return LD_OK;
}

/* calc_Parameters, L_CUDA.cu:267-278 */
ld_status ld_problem_check_launch(ld_problem *p, int32_t blocks, int32_t threads) {
    if (!p) return ld_fail(LD_ERR_ARG, "null argument");
    uint64_t total = p->labelings;
    if ((uint64_t)threads > total) threads = (int32_t)total;
    if (threads == 0) blocks = 0;
    else if (total / (uint64_t)threads < (uint64_t)blocks) blocks = (int32_t)(total / (uint64_t)threads);
    ld_logf(p, "num_ofBlock: %d, num_ofThread in block: %d\n", blocks, threads);
    ld_logf(p, "maximum length of strategy vector: %d\n", p->max_rows);
    if (p->max_rows < p->R) {
        ld_logf(p, "Matrix is too large. The matrix has %d rows after reduction. The maximum number of rows cannot be more than %d.\n", p->R, p->max_rows);
        return ld_fail(LD_ERR_LIMIT, "%d reduced rows exceed the maximum %d", p->R, p->max_rows);
    }
    if (p->C > LD_MAX_COLS) {
        ld_logf(p, "Matrix is too large. The length variable %d should be greater or equal than %d.\n", LD_MAX_COLS, p->C);
        return ld_fail(LD_ERR_LIMIT, "%d reduced columns exceed %d", p->C, LD_MAX_COLS);
    }
    return LD_OK;
}

ld_status ld_gray_labels(uint64_t index, int32_t rows, int32_t d, int32_t *labels) {
    if (!labels && rows > 1) return ld_fail(LD_ERR_ARG, "null labels");
    if (d <= 2) {
        uint64_t g = index ^ (index >> 1);
        for (int i = 0; i < rows - 1; i++) labels[i] = (int32_t)((g >> i) & 1u);
        return LD_OK;
    }
    uint64_t q = index;
    for (int i = 0; i < rows - 1; i++) {
        uint64_t r = q % (uint64_t)(2 * d);
        labels[i] = (int32_t)(r < (uint64_t)d ? r : (uint64_t)(2 * d - 1) - r);
        q /= (uint64_t)d;
    }
    return LD_OK;
}

ld_status ld_problem_solve(ld_problem *p, const ld_options *opt, ld_result *res) {
    if (!p || !res) return ld_fail(LD_ERR_ARG, "null argument");
    if (p->R == 0) {
        memset(res, 0, sizeof *res);
        res->kernel_kind = LD_KERNEL_NONE;
        return LD_OK;
    }
    return ld_solve_reduced(p->red, p->R, p->C, p->d, p->marg, opt, res, NULL);
}

/* print_results, functions.h:371-412 */
ld_status ld_problem_report(ld_problem *p, const ld_result *res, int32_t *strategy,
                            int32_t cap, int32_t *count, char *name, size_t name_cap) {
    if (!p || !res) return ld_fail(LD_ERR_ARG, "null argument");
    if (p->d_user == 1 && p->marg_user) {
        ld_logf(p, "LM is: %lld\n", (long long)res->value);
        if (name) snprintf(name, name_cap, "strategy_LM.txt");
    } else {
        ld_logf(p, "L%d is: %lld\n", p->d_user, (long long)res->value);
        if (name) snprintf(name, name_cap, "strategy_L%d.txt", p->d_user);
    }
    if (cap < p->orig_len) return ld_fail(LD_ERR_ARG, "strategy buffer holds %d, need %d", cap, p->orig_len);
    int32_t lab[LD_INDEX_BITS] = {0};
    if (p->R > 0) ld_gray_labels(res->gray_index, p->R, p->d, lab);
    int fixed = p->d == 1 ? 1 : 0;
    int j = 0;
    int *val = (int *)calloc((size_t)(p->orig_len > 0 ? p->orig_len : 1), sizeof(int));
    if (!val) return ld_fail(LD_ERR_NOMEM, "out of host memory");
    for (int i = 0; i < p->orig_len; i++) {
        int m = p->orig[i], v;
        if (m == 0) {                       /* a kept line */
            if (p->marg && p->d == 1) {
                v = (j == 0) ? 1 : (j == p->R - 1 ? lab[0] : lab[j]);
            } else {
                v = (j == p->R - 1) ? fixed : lab[j];
            }
            j++;
        } else if (m == p->orig_len) {      /* a zero line */
            v = fixed;
        } else if (m < 0) {                 /* united with opposite sign */
            v = (val[-m - 1] + 1) & 1;
        } else {                            /* united with the same sign */
            v = val[m - 1];
        }
        val[i] = v;
        if (strategy) strategy[i] = p->d == 1 ? 2 * v - 1 : v;
    }
    free(val);
    if (count) *count = p->orig_len;
    return LD_OK;
}
