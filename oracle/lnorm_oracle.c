/*
 * lnorm_oracle.c -- TEST INFRASTRUCTURE ONLY (see lnorm_oracle.h).
 *
 * CPU restatement of the reference's brute-force L_d solver.  Each
 * function names the reference lines it restates.  Written for clarity,
 * not speed, except the enumeration loop which must cover ~1e9 labelings
 * in seconds; it is OpenMP-parallel over contiguous Gray-index ranges
 * exactly like the reference's worker split (L_CUDA.cu:5-12).
 */
#include "lnorm_oracle.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_LENGTH 4096      /* functions.h:2   max columns            */
#define OR_RANK 10          /* functions.h:3   max order d            */
#define OR_BITS 64          /* functions.h:4   bits of the Gray index */

/* ------------------------------------------------------------------ */
/* growable text buffer for the stdout lines                           */
typedef struct { char *p; size_t n, cap; } sbuf;
static void sb_printf(sbuf *b, const char *fmt, ...)
    __attribute__((format(printf, 2, 3)));
#include <stdarg.h>
static void sb_printf(sbuf *b, const char *fmt, ...) {
    va_list ap; char tmp[512];
    va_start(ap, fmt); int k = vsnprintf(tmp, sizeof tmp, fmt, ap); va_end(ap);
    if (k < 0) return;
    if (b->n + (size_t)k + 1 > b->cap) {
        size_t nc = (b->cap + (size_t)k + 1) * 2;
        b->p = (char *)realloc(b->p, nc); b->cap = nc;
    }
    memcpy(b->p + b->n, tmp, (size_t)k); b->n += (size_t)k; b->p[b->n] = 0;
}

/* ------------------------------------------------------------------ */
/* state: the reference's `item` / `item_calc` (functions.h:7-38)       */
typedef struct {
    int R0, C0;          /* rows / cols as read                        */
    int64_t *a;          /* R0*C0 working matrix, mutated by uniting   */
    int *mr, *mc;        /* original_r / original_c markers            */
    int R, C;            /* iRows_reduced / iCols_reduced              */
    int d_user, d_eff;   /* n_original / n                             */
    char stat;
    int marg_user;       /* first->marginal                            */
    int marg;            /* second->marginal                           */
    int transposed;
    int *orig; int orig_len;   /* first->original / original_length    */
    int64_t *red;        /* mtx_as_vec                                 */
    sbuf log;
} or_state;

#define A(s, i, j) ((s)->a[(size_t)(i) * (s)->C0 + (j)])

static int is_prep(char c) {
    return c == 'y' || c == 'Y' || c == 'r' || c == 'R' || c == 'c' || c == 'C';
}
static int is_rows(char c) { return c == 'y' || c == 'Y' || c == 'r' || c == 'R'; }
static int is_cols(char c) { return c == 'y' || c == 'Y' || c == 'c' || c == 'C'; }

/* matrix_read, functions.h:40-79.  Token characters are 0-9 e E . + -;
 * any other byte ends a token; '\n' or end of input ends a row when the
 * row has entries.  Tokens with e/E go through %le and are truncated,
 * others through %d (here %lld: int64 input).  A token scanf cannot
 * convert leaves the previous value in place, as the reference's local
 * variable does.  The column count is the last row's entry count;
 * shorter rows would be read out of bounds by the reference (undefined),
 * so they are rejected (-2). */
static int or_parse(or_state *s, const char *text, size_t len) {
    char tok[256]; int ti = 0, has_e = 0;
    int64_t value = 0; double dv;
    int64_t *row = NULL; int j = 0, cap_row = 0;
    int64_t **rows = NULL; int *rlen = NULL; int k = 0, cap_rows = 0;
    int cols = 0;
    for (size_t p = 0; p <= len; p++) {
        int eof = (p == len);
        char g = eof ? 0 : text[p];
        if (!eof && ((g >= '0' && g <= '9') || g == 'e' || g == 'E' || g == '.' || g == '+' || g == '-')) {
            if (ti < 255) tok[ti++] = g;
            if (g == 'e' || g == 'E') has_e = 1;
            continue;
        }
        tok[ti] = 0;
        if (tok[0] != 0) {
            if (has_e) { if (sscanf(tok, "%le", &dv) == 1) value = (int64_t)dv; has_e = 0; }
            else { long long v; if (sscanf(tok, "%lld", &v) == 1) value = v; }
            if (j == cap_row) { cap_row = cap_row ? 2 * cap_row : 16; row = (int64_t *)realloc(row, cap_row * sizeof *row); }
            row[j++] = value;
            ti = 0;
        }
        tok[0] = 0;
        if ((eof || g == '\n') && j > 0) {
            if (k == cap_rows) {
                cap_rows = cap_rows ? 2 * cap_rows : 16;
                rows = (int64_t **)realloc(rows, cap_rows * sizeof *rows);
                rlen = (int *)realloc(rlen, cap_rows * sizeof *rlen);
            }
            rows[k] = row; rlen[k] = j; cols = j; k++;
            row = NULL; cap_row = 0; j = 0;
        }
    }
    free(row);
    int bad = (k == 0);
    for (int i = 0; i < k && !bad; i++) if (rlen[i] < cols) bad = 1;
    if (!bad) {
        s->R0 = k; s->C0 = cols;
        s->a = (int64_t *)malloc((size_t)k * cols * sizeof(int64_t));
        for (int i = 0; i < k; i++) memcpy(s->a + (size_t)i * cols, rows[i], cols * sizeof(int64_t));
        sb_printf(&s->log, "rows: %d, cols: %d\n", k, cols);
    }
    for (int i = 0; i < k; i++) free(rows[i]);
    free(rows); free(rlen);
    return bad ? -2 : 0;
}

/* eliminate_zero_rows_cols, functions.h:109-151. */
static void or_zero_lines(or_state *s) {
    s->mr = (int *)calloc(s->R0, sizeof(int));
    s->mc = (int *)calloc(s->C0, sizeof(int));
    s->R = s->R0; s->C = s->C0; s->marg = s->marg_user;
    if (!is_prep(s->stat)) return;
    int cr = 0, cc = 0;
    for (int i = 0; i < s->R0; i++) {
        int zero = 1;
        for (int k = 0; k < s->C0 && zero; k++) if (A(s, i, k) != 0) zero = 0;
        if (zero) {
            s->mr[i] = s->R0;
            if (s->marg_user == 0 || i > 0) { cr++; sb_printf(&s->log, "row %d entries are zeros.\n", i + 1); }
        }
    }
    s->R = s->R0 - cr;
    for (int i = 0; i < s->C0; i++) {
        int zero = 1;
        for (int k = 0; k < s->R0 && zero; k++) if (A(s, k, i) != 0) zero = 0;
        if (zero) {
            s->mc[i] = s->C0;
            if (s->marg_user == 0 || i > 0) { cc++; sb_printf(&s->log, "col %d entries are zeros.\n", i + 1); }
        }
    }
    s->C = s->C0 - cc;
    if (s->marg_user == 1) {
        if (s->mr[0] == s->R0 && s->mc[0] == s->C0) {
            s->marg = 0; s->R--; s->C--;
            sb_printf(&s->log, "The entries of the first row and column are zeros.\n");
        } else { s->mr[0] = 0; s->mc[0] = 0; }
    }
}

/* proportionality test of two lines, functions.h:248-255 (rows) and
 * 275-282 (cols): first position where not both are zero is the pivot;
 * a zero/nonzero mismatch there, or any unequal cross product after it,
 * means "not proportional".  Returns 0 (no), 1 (parallel), -1 (anti). */
static int or_prop(const int64_t *x, const int64_t *y, int n, size_t stride) {
    int k = 0;
    while (k < n && x[k * stride] == 0 && y[k * stride] == 0) k++;
    if (k == n) return 0;
    if ((x[k * stride] == 0) != (y[k * stride] == 0)) return 0;
    int piv = k;
    for (; k < n - 1; k++) {
        __int128 m1 = (__int128)x[piv * stride] * y[(k + 1) * stride];
        __int128 m2 = (__int128)y[piv * stride] * x[(k + 1) * stride];
        if (m1 != m2) return 0;
    }
    __int128 pp = (__int128)x[piv * stride] * y[piv * stride];
    return pp < 0 ? -1 : 1;
}

/* calc_reduce_matrix_rows, functions.h:237-262.  Anti-parallel rows are
 * united only for d == 1 (line 257). */
static void or_unite_rows(or_state *s) {
    int cnt = 0;
    for (int i = s->marg_user; i < s->R0; i++) {
        if (s->mr[i] != 0) continue;
        for (int j = i + 1; j < s->R0; j++) {
            if (s->mr[j] != 0) continue;
            int p = or_prop(&A(s, i, 0), &A(s, j, 0), s->C0, 1);
            if (p == 0) continue;
            if (p < 0) {
                if (s->d_user == 1) {
                    s->mr[j] = -(i + 1); cnt++;
                    for (int k = 0; k < s->C0; k++) A(s, i, k) -= A(s, j, k);
                    sb_printf(&s->log, "row %d was subtracted from %d\n", j + 1, i + 1);
                }
            } else {
                s->mr[j] = i + 1; cnt++;
                for (int k = 0; k < s->C0; k++) A(s, i, k) += A(s, j, k);
                sb_printf(&s->log, "row %d was added to %d\n", j + 1, i + 1);
            }
        }
    }
    s->R -= cnt;
}

/* calc_reduce_matrix_cols, functions.h:264-289 (anti-parallel united for
 * every d, line 284). */
static void or_unite_cols(or_state *s) {
    int cnt = 0;
    for (int i = s->marg_user; i < s->C0; i++) {
        if (s->mc[i] != 0) continue;
        for (int j = i + 1; j < s->C0; j++) {
            if (s->mc[j] != 0) continue;
            int p = or_prop(&A(s, 0, i), &A(s, 0, j), s->R0, (size_t)s->C0);
            if (p == 0) continue;
            if (p < 0) {
                s->mc[j] = -(i + 1); cnt++;
                for (int k = 0; k < s->R0; k++) A(s, k, i) -= A(s, k, j);
                sb_printf(&s->log, "col %d was subtracted from %d\n", j + 1, i + 1);
            } else {
                s->mc[j] = i + 1; cnt++;
                for (int k = 0; k < s->R0; k++) A(s, k, i) += A(s, k, j);
                sb_printf(&s->log, "col %d was added to %d\n", j + 1, i + 1);
            }
        }
    }
    s->C -= cnt;
}

/* calc_reduce_matrix_cols_sign, functions.h:193-235 (d > 1 only): every
 * single-signed surviving column is folded into the first one. */
static void or_sign_cols(or_state *s) {
    int *sg = (int *)calloc(s->C0, sizeof(int));
    int cnt = 0;
    for (int c = 0; c < s->C0; c++) {
        if (s->mc[c] != 0) continue;
        int pos = 0, neg = 0;
        for (int k = 0; k < s->R0 && (!pos || !neg); k++) {
            if (A(s, k, c) > 0) pos = 1;
            if (A(s, k, c) < 0) neg = 1;
        }
        if (pos && neg) sg[c] = 0;
        else if (neg) { sg[c] = -1; cnt++; }
        else { sg[c] = 1; cnt++; }
    }
    if (cnt > 1) {
        s->C -= cnt - 1;
        int f = 0; while (sg[f] == 0) f++;
        for (int c = f + 1; c < s->C0; c++) {
            if (s->mc[c] != 0) continue;
            int p = sg[f] * sg[c];
            if (p < 0) {
                s->mc[c] = -(f + 1);
                for (int k = 0; k < s->R0; k++) A(s, k, f) -= A(s, k, c);
                sb_printf(&s->log, "col %d was subtracted from %d\n", c + 1, f + 1);
            }
            if (p > 0) {
                s->mc[c] = f + 1;
                for (int k = 0; k < s->R0; k++) A(s, k, f) += A(s, k, c);
                sb_printf(&s->log, "col %d was added to %d\n", c + 1, f + 1);
            }
        }
    }
    free(sg);
}

/* delete_rows / delete_cols (functions.h:153-191) keep the surviving
 * lines in their original order; convert_mtx_to_vec (functions.h:291-329)
 * flattens, transposes for d == 1 with more rows than columns, and swaps
 * the marginal row to the last (fixed) position. */
static void or_flatten(or_state *s) {
    int *ri = (int *)malloc(sizeof(int) * (s->R0 + 1));
    int *ci = (int *)malloc(sizeof(int) * (s->C0 + 1));
    int nr = 0, nc = 0;
    for (int i = 0; i < s->R0; i++) if (!is_prep(s->stat) || s->mr[i] == 0) ri[nr++] = i;
    for (int i = 0; i < s->C0; i++) if (!is_prep(s->stat) || s->mc[i] == 0) ci[nc++] = i;
    /* the reduced counts and the survivors agree by construction */
    if (nr > s->R) nr = s->R;
    if (nc > s->C) nc = s->C;
    s->red = (int64_t *)calloc((size_t)(s->R > 0 ? s->R : 1) * (s->C > 0 ? s->C : 1), sizeof(int64_t));
    if (s->d_user == 1 && s->R > s->C) {
        for (int j = 0; j < s->C; j++)
            for (int i = 0; i < s->R; i++)
                s->red[(size_t)j * s->R + i] = A(s, ri[i], ci[j]);
        int t = s->R; s->R = s->C; s->C = t;
        s->orig = s->mc; s->orig_len = s->C0; s->transposed = 1;
        sb_printf(&s->log, "Matrix was transposed.\n");
    } else {
        for (int i = 0; i < s->R; i++)
            for (int j = 0; j < s->C; j++)
                s->red[(size_t)i * s->C + j] = A(s, ri[i], ci[j]);
        s->orig = s->mr; s->orig_len = s->R0; s->transposed = 0;
    }
    if (s->marg == 1 && s->R > 0) {
        for (int j = 0; j < s->C; j++) {
            int64_t t = s->red[(size_t)(s->R - 1) * s->C + j];
            s->red[(size_t)(s->R - 1) * s->C + j] = s->red[j];
            s->red[j] = t;
        }
    }
    free(ri); free(ci);
}

uint64_t or_total(int rows, int d) {
    if (rows <= 0) return 0;
    if (d <= 2) return (uint64_t)1 << (rows - 1);
    uint64_t t = 1;
    for (int i = 0; i < rows - 1; i++) t *= (uint64_t)d;
    return t;
}

/* calc_Parameters, L_CUDA.cu:242-279: d reset, work count, launch clamp,
 * limits.  Returns -1 on the reference's exit(-1) paths. */
static int or_params(or_state *s, int blocks, int threads) {
    if (s->d_user < s->R || s->d_user == 1) s->d_eff = s->d_user;
    else {
        s->d_eff = s->R > 1 ? s->R : 2;
        sb_printf(&s->log, "The preprocessed matrix has a number of rows (%d) less than or equal to the order of the L norm (%d).\n", s->R, s->d_user);
    }
    uint64_t total = or_total(s->R, s->d_eff);
    int maxRows = s->d_eff <= 2 ? OR_BITS - 1 : (int)(floor(OR_BITS / log2(s->d_eff)) + 1);
    if ((uint64_t)threads > total) threads = (int)total;
    if (threads == 0) blocks = 0;
    else if (total / (uint64_t)threads < (uint64_t)blocks) blocks = (int)(total / (uint64_t)threads);
    sb_printf(&s->log, "num_ofBlock: %d, num_ofThread in block: %d\n", blocks, threads);
    sb_printf(&s->log, "maximum length of strategy vector: %d\n", maxRows);
    if (maxRows < s->R) {
        sb_printf(&s->log, "Matrix is too large. The matrix has %d rows after reduction. The maximum number of rows cannot be more than %d.\n", s->R, maxRows);
        return -1;
    }
    if (s->C > OR_LENGTH) {
        sb_printf(&s->log, "Matrix is too large. The length variable %d should be greater or equal than %d.\n", OR_LENGTH, s->C);
        return -1;
    }
    return 0;
}

static int or_prepare(or_state *s, const char *text, size_t len, int d, char stat, int marginal) {
    memset(s, 0, sizeof *s);
    s->d_user = d; s->stat = stat; s->marg_user = (d == 1) ? marginal : 0;
    int rc = or_parse(s, text, len);
    if (rc) return rc;
    or_zero_lines(s);
    if (is_rows(stat)) or_unite_rows(s);
    if (is_cols(stat)) { or_unite_cols(s); if (d > 1) or_sign_cols(s); }
    or_flatten(s);
    return 0;
}

static void or_free(or_state *s) {
    free(s->a); free(s->mr); free(s->mc); free(s->red); free(s->log.p);
}

/* ------------------------------------------------------------------ */
/* Gray codes.  Binary reflected: label_i(N) = ((N + 2^i) >> (i+1)) & 1
 * (L_CUDA.cu:61-63).  d-ary reflected: label_i(N) =
 * pattern[(N / d^i) mod 2d], pattern = 0..d-1,d-1..0 (functions.h:350-369,
 * L_CUDA.cu:204-206). */
void or_labels(uint64_t N, int rows, int d, int32_t *lab) {
    if (d <= 2) {
        for (int i = 0; i < rows - 1; i++) lab[i] = (int32_t)(((N + ((uint64_t)1 << i)) >> (i + 1)) & 1u);
        return;
    }
    uint64_t q = N;
    for (int i = 0; i < rows - 1; i++) {
        uint64_t r = q % (uint64_t)(2 * d);
        lab[i] = (int32_t)(r < (uint64_t)d ? r : (uint64_t)(2 * d) - 1 - r);
        q /= (uint64_t)d;
    }
}

int64_t or_value(const int64_t *a, int R, int C, int d, int marginal, const int32_t *lab) {
    int nv = d <= 1 ? 1 : d;
    int64_t *v = (int64_t *)calloc((size_t)nv * C, sizeof(int64_t));
    for (int l = 0; l < C; l++) v[l] = a[(size_t)(R - 1) * C + l];   /* fixed row: +1 / message 0 */
    for (int i = 0; i < R - 1; i++) {
        if (d <= 1) { int64_t sg = lab[i] ? 1 : -1; for (int l = 0; l < C; l++) v[l] += sg * a[(size_t)i * C + l]; }
        else { for (int l = 0; l < C; l++) v[(size_t)lab[i] * C + l] += a[(size_t)i * C + l]; }
    }
    int64_t sum = 0;
    for (int m = 0; m < nv; m++)
        for (int l = 0; l < C; l++) {
            int64_t x = v[(size_t)m * C + l];
            sum += (d <= 1 && marginal && l == 0) ? x : (x < 0 ? -x : x);
        }
    free(v);
    return sum;
}

/* One worker's contiguous Gray range [lo, hi): seed from the direct
 * labels of lo, then walk.  Per step exactly one row changes label
 * (L_CUDA.cu:72-84 for d==1, 111-123 d==2, 160-182 d==3, 218-238 d>=4);
 * the row is the lowest base-d position whose digit of N is nonzero.
 * The first (smallest) N attaining the range's maximum is kept, as the
 * reference's strict '>' does. */
static void or_walk(const int64_t *a, int R, int C, int d, int marginal,
                    uint64_t lo, uint64_t hi, int64_t *best, uint64_t *bestN) {
    int nv = d <= 1 ? 1 : d;
    int dd = d <= 2 ? 2 : d;
    int32_t lab[OR_BITS];
    int64_t *v = (int64_t *)calloc((size_t)nv * C, sizeof(int64_t));
    or_labels(lo, R, d, lab);
    for (int l = 0; l < C; l++) v[l] = a[(size_t)(R - 1) * C + l];
    for (int i = 0; i < R - 1; i++) {
        if (d <= 1) { int64_t sg = lab[i] ? 1 : -1; for (int l = 0; l < C; l++) v[l] += sg * a[(size_t)i * C + l]; }
        else for (int l = 0; l < C; l++) v[(size_t)lab[i] * C + l] += a[(size_t)i * C + l];
    }
    /* base-d digits of N for the change search, and the parity of their sum
     * (for odd d the parity of a number equals the parity of its digit sum) */
    int dig[OR_BITS + 1];
    int dsum = 0;
    { uint64_t q = lo; for (int i = 0; i <= OR_BITS; i++) { dig[i] = (int)(q % (uint64_t)dd); dsum ^= dig[i] & 1; q /= (uint64_t)dd; } }
    int64_t bv = 0; uint64_t bn = lo; int first = 1;
    for (uint64_t N = lo; N < hi; N++) {
        if (N != lo) {
            /* increment the base-d counter; i = lowest digit that did not wrap */
            int i = 0;
            while (dig[i] == dd - 1) { dig[i] = 0; i++; }
            dig[i]++;
            dsum ^= 1;   /* used for odd d only: a wrap (d-1 -> 0) keeps the parity */
            /* new label of row i = pattern[(N / d^i) mod 2d]: digit i itself when
             * floor(N / d^(i+1)) is even, reflected (d-1-digit) when odd */
            int newl;
            if (d <= 2) newl = lab[i] ^ 1;
            else {
                int par;   /* parity of floor(N / d^(i+1)) */
                if (dd & 1) par = (dsum ^ dig[i]) & 1;   /* digits below i are 0 now */
                else par = dig[i + 1] & 1;
                newl = par ? dd - 1 - dig[i] : dig[i];
            }
            const int64_t *row = a + (size_t)i * C;
            if (d <= 1) {
                int64_t sg = newl ? 2 : -2;
                for (int l = 0; l < C; l++) v[l] += sg * row[l];
            } else {
                int o = lab[i];
                for (int l = 0; l < C; l++) { v[(size_t)o * C + l] -= row[l]; v[(size_t)newl * C + l] += row[l]; }
            }
            lab[i] = newl;
        }
        int64_t sum = 0;
        for (int m = 0; m < nv; m++)
            for (int l = 0; l < C; l++) {
                int64_t x = v[(size_t)m * C + l];
                sum += (d <= 1 && marginal && l == 0) ? x : (x < 0 ? -x : x);
            }
        if (first || sum > bv) { bv = sum; bn = N; first = 0; }
    }
    free(v);
    *best = bv; *bestN = bn;
}

int or_enumerate(const int64_t *a, int R, int C, int d, int marginal,
                 uint64_t lo, uint64_t hi, int nthreads,
                 int64_t *value, uint64_t *index) {
    if (R <= 0 || C <= 0) { *value = 0; *index = 0; return 0; }
    uint64_t total = or_total(R, d);
    if (hi == 0 || hi > total) hi = total;
    if (lo >= hi) return -1;
    if (nthreads < 1) nthreads = 1;
    uint64_t n = hi - lo;
    if ((uint64_t)nthreads > n) nthreads = (int)n;
    int64_t *bv = (int64_t *)malloc(sizeof(int64_t) * nthreads);
    uint64_t *bn = (uint64_t *)malloc(sizeof(uint64_t) * nthreads);
    uint64_t steps = n / (uint64_t)nthreads, rem = n % (uint64_t)nthreads;
#pragma omp parallel for num_threads(nthreads) schedule(static, 1)
    for (int w = 0; w < nthreads; w++) {
        /* calc_jmin_jmax, L_CUDA.cu:5-12 */
        uint64_t wl = lo + (uint64_t)w * steps + ((uint64_t)w < rem ? (uint64_t)w : rem);
        uint64_t wh = wl + steps + ((uint64_t)w < rem ? 1 : 0);
        or_walk(a, R, C, d, marginal, wl, wh, &bv[w], &bn[w]);
    }
    /* host argmax with strict '<': the lowest worker wins ties (L_CUDA.cu:345-348) */
    int64_t v = bv[0]; uint64_t N = bn[0];
    for (int w = 1; w < nthreads; w++) if (bv[w] > v) { v = bv[w]; N = bn[w]; }
    free(bv); free(bn);
    *value = v; *index = N;
    return 0;
}

int or_preprocess(const char *text, size_t len, int d, char stat, int marginal,
                  int64_t *red, size_t cap, int *rows, int *cols,
                  int *d_eff, int *marginal_eff, int *transposed) {
    or_state s;
    int rc = or_prepare(&s, text, len, d, stat, marginal);
    if (rc == 0) rc = or_params(&s, 1, 1);
    if (rc == 0 || rc == -1) {
        *rows = s.R; *cols = s.C; *d_eff = s.d_eff; *marginal_eff = s.marg; *transposed = s.transposed;
        if ((size_t)s.R * s.C <= cap && s.R > 0) memcpy(red, s.red, (size_t)s.R * s.C * sizeof(int64_t));
    }
    or_free(&s);
    return rc;
}

/* print_results, functions.h:371-412: value line and the strategy file in
 * the original indexing (kept lines take their solved label, the marginal
 * row +1, zero lines the default label, united lines the label of the line
 * they were united into, negated for subtraction). */
static void or_results(or_state *s, int64_t value, const int32_t *strat, sbuf *file, char *name, size_t cap_name) {
    if (s->d_user == 1 && s->marg_user == 1) {
        sb_printf(&s->log, "LM is: %lld\n", (long long)value);
        snprintf(name, cap_name, "strategy_LM.txt");
    } else {
        sb_printf(&s->log, "L%d is: %lld\n", s->d_user, (long long)value);
        snprintf(name, cap_name, "strategy_L%d.txt", s->d_user);
    }
    int *out = (int *)calloc(s->orig_len > 0 ? s->orig_len : 1, sizeof(int));
    int j = 0;
    for (int i = 0; i < s->orig_len; i++) {
        int val, m = s->orig[i];
        if (m == 0) {
            if (s->marg == 1 && s->d_eff == 1) {
                if (j == 0) val = 1;
                else if (j == s->R - 1) val = strat[0];
                else val = strat[j];
            } else {
                if (j == s->R - 1) val = s->d_eff == 1 ? 1 : 0;
                else val = strat[j];
            }
            j++;
        } else if (m == s->orig_len) val = s->d_eff == 1 ? 1 : 0;
        else if (m < 0) val = (out[-m - 1] + 1) & 1;
        else val = out[m - 1];
        out[i] = val;
        sb_printf(file, "%d\n", s->d_eff == 1 ? 2 * val - 1 : val);
    }
    free(out);
}

static void copy_out(const sbuf *b, char *dst, size_t cap) {
    if (!dst || cap == 0) return;
    size_t n = b->n < cap - 1 ? b->n : cap - 1;
    if (b->p) memcpy(dst, b->p, n);
    dst[n] = 0;
}

int or_run_cli(const char *text, size_t len, int blocks, int threads, int d,
               char stat, int marginal, int nthreads,
               char *out_stdout, size_t cap_stdout,
               char *out_strategy, size_t cap_strategy,
               char *strategy_name, size_t cap_name, int64_t *value_out) {
    or_state s;
    int rc = or_prepare(&s, text, len, d, stat, marginal);
    if (rc == 0) rc = or_params(&s, blocks, threads);
    if (rc != 0) { copy_out(&s.log, out_stdout, cap_stdout); or_free(&s); return rc; }
    int64_t value = 0; uint64_t N = 0;
    int32_t strat[OR_BITS] = {0};
    if (s.R == 0) sb_printf(&s.log, "This is a zero matrix.\n");
    else {
        or_enumerate(s.red, s.R, s.C, s.d_eff, s.marg, 0, 0, nthreads, &value, &N);
        or_labels(N, s.R, s.d_eff, strat);
    }
    sbuf file = {0};
    or_results(&s, value, strat, &file, strategy_name, cap_name);
    copy_out(&s.log, out_stdout, cap_stdout);
    copy_out(&file, out_strategy, cap_strategy);
    if (value_out) *value_out = value;
    free(file.p);
    or_free(&s);
    return 0;
}
