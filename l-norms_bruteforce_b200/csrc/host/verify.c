/*
 * Strategy verifier (no counterpart in the reference): the value, on the
 * matrix as read, of the labeling a strategy file records.  The file is the
 * one print_results writes (functions.h:371-412): one entry per line of the
 * input (per row, or per column when the d = 1 problem was transposed,
 * L_CUDA.cu:417-421), +1/-1 for d = 1 and 0..d-1 otherwise, united and zero
 * lines included.
 *
 *   d = 1:   sum over the other lines l of |sum_i s_i A(i, l)|; with the
 *            marginal flag the l = 0 term (the marginal row or column) is
 *            the signed sum itself (the LM kernel, L_CUDA.cu:14-49);
 *   d >= 2:  sum over labels k and lines l of |sum over i labelled k of A(i, l)|.
 *
 * The sums are exact (128-bit accumulation, LD_ERR_LIMIT beyond 64 bits).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ld_internal.h"

static int64_t entry(const int64_t *a, int R0, int C0, int transposed, int i, int l) {
    (void)R0;
    return transposed ? a[(size_t)l * C0 + i] : a[(size_t)i * C0 + l];
}

ld_status ld_strategy_value(const char *text, size_t len, int32_t d, char stat, int32_t marginal,
                            const int32_t *strategy, int32_t count, int64_t *value) {
    if (!text || !strategy || !value) return ld_fail(LD_ERR_ARG, "null argument");
    if (d < 1 || d > LD_MAX_D) return ld_fail(LD_ERR_ARG, "order d=%d outside 1..%d", d, LD_MAX_D);
    int64_t *a = NULL;
    int R0 = 0, C0 = 0;
    ld_status st = ld_parse_matrix_text(text, len, &a, &R0, &C0);
    if (st != LD_OK) return st;
    /* the orientation the solver labelled: the same preprocessing */
    int64_t *copy = (int64_t *)malloc((size_t)R0 * C0 * sizeof(int64_t));
    if (!copy) { free(a); return ld_fail(LD_ERR_NOMEM, "out of host memory"); }
    memcpy(copy, a, (size_t)R0 * C0 * sizeof(int64_t));
    ld_problem *p = NULL;
    st = ld_problem_build(copy, R0, C0, d, stat, marginal, &p);
    if (st != LD_OK) { free(a); return st; }
    const int transposed = p->transposed, lm = p->marg_user;
    ld_problem_destroy(p);
    const int lines = transposed ? C0 : R0, other = transposed ? R0 : C0;
    if (count != lines) {
        free(a);
        return ld_fail(LD_ERR_ARG, "strategy has %d entries, the %s number %d", count,
                       transposed ? "columns" : "rows", lines);
    }
    for (int i = 0; i < lines; i++) {
        const int v = strategy[i];
        if (d == 1 ? (v != 1 && v != -1) : (v < 0 || v >= d)) {
            free(a);
            return ld_fail(LD_ERR_ARG, "strategy entry %d is %d", i + 1, v);
        }
    }
    const int nlab = d == 1 ? 1 : d;
    __int128 total = 0;
    for (int k = 0; k < nlab; k++) {
        for (int l = 0; l < other; l++) {
            __int128 s = 0;
            for (int i = 0; i < lines; i++) {
                const int64_t x = entry(a, R0, C0, transposed, i, l);
                if (d == 1) s += strategy[i] > 0 ? (__int128)x : -(__int128)x;
                else if (strategy[i] == k) s += x;
            }
            total += (d == 1 && lm && l == 0) ? s : (s < 0 ? -s : s);
        }
    }
    free(a);
    if (total > (__int128)INT64_MAX || total < (__int128)INT64_MIN)
        return ld_fail(LD_ERR_LIMIT, "the value exceeds 64 bits");
    *value = (int64_t)total;
    return LD_OK;
}

static char *read_all(const char *path, size_t *len) {
    FILE *f = fopen(path, "rb");
    if (!f) return NULL;
    size_t cap = 1 << 16, n = 0;
    char *buf = (char *)malloc(cap + 1);
    while (buf) {
        const size_t k = fread(buf + n, 1, cap - n, f);
        n += k;
        if (n < cap) break;
        cap *= 2;
        char *nb = (char *)realloc(buf, cap + 1);
        if (!nb) free(buf);
        buf = nb;
    }
    fclose(f);
    if (buf) { buf[n] = 0; *len = n; }
    return buf;
}

/* `L_verify matrix_file strategy_file d [y|c|r] [m]`: prints the value line
 * the solver prints ("L3 is: 258", "LM is: 398") for the strategy's
 * labeling; exit status 0, or 1 with a message on stderr. */
int ld_verify_main(int argc, char **argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s matrix_file strategy_file d [y|c|r] [m]\n", argc > 0 ? argv[0] : "L_verify");
        return 1;
    }
    /* the optional arguments as arguments_CUDA reads them (L_CUDA.cu:392-409):
     * the first is the preprocessing flag, the marginal flag is the last one
     * given (d = 1 only) */
    const int d = atoi(argv[3]);
    const char stat = argc > 4 ? argv[4][0] : 'n';
    const char *mflag = argc > 5 ? argv[5] : (argc > 4 ? argv[4] : "");
    const int marginal = d == 1 && (mflag[0] == 'm' || mflag[0] == 'M');
    size_t mlen = 0, slen = 0;
    char *mtext = read_all(argv[1], &mlen);
    if (!mtext) { fprintf(stderr, "cannot open %s\n", argv[1]); return 1; }
    char *stext = read_all(argv[2], &slen);
    if (!stext) { free(mtext); fprintf(stderr, "cannot open %s\n", argv[2]); return 1; }
    size_t cap = 64, n = 0;
    int32_t *lab = (int32_t *)malloc(cap * sizeof(int32_t));
    char *s = stext, *end = NULL;
    for (;;) {
        if (!lab) break;
        const long v = strtol(s, &end, 10);
        if (end == s) break;
        if (n == cap) {
            cap *= 2;
            int32_t *nl = (int32_t *)realloc(lab, cap * sizeof(int32_t));
            if (!nl) free(lab);
            lab = nl;
            if (!lab) break;
        }
        lab[n++] = (int32_t)v;
        s = end;
    }
    int rc = 1;
    int64_t value = 0;
    if (!lab) fprintf(stderr, "out of host memory\n");
    else if (ld_strategy_value(mtext, mlen, d, stat, marginal, lab, (int32_t)n, &value) != LD_OK)
        fprintf(stderr, "%s\n", ld_last_error());
    else {
        if (d == 1 && marginal) printf("LM is: %lld\n", (long long)value);
        else printf("L%d is: %lld\n", d, (long long)value);
        rc = 0;
    }
    free(lab);
    free(stext);
    free(mtext);
    return rc;
}
