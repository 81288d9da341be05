/*
 * Matrix text reader: the input contract of matrix_read (functions.h:40-79).
 *
 *  - Entry characters are 0-9 e E . + - ; any other byte separates entries.
 *  - '\n' (or the end of the text) closes a row that has entries; rows with
 *    no entries (blank lines) are skipped.
 *  - An entry containing e/E is read with %le and truncated toward zero
 *    (scientific notation such as 3.10000000e+01); other entries with %d
 *    semantics (here 64-bit: sign, digits, stop at the first other char).
 *  - An entry scanf cannot convert (e.g. "-" or ".") repeats the previous
 *    entry's value, which is what the reference's reused local does.
 *  - The column count is the entry count of the LAST row; longer rows are
 *    truncated to it.  Shorter rows are rejected: the reference would read
 *    past their end (undefined behaviour).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ld_internal.h"

static int is_entry_char(char g) {
    return (g >= '0' && g <= '9') || g == 'e' || g == 'E' || g == '.' || g == '+' || g == '-';
}

ld_status ld_parse_matrix_text(const char *text, size_t len, int64_t **out, int *rows, int *cols) {
    /* entries are appended to one flat buffer; row ends are recorded */
    size_t cap = 256, n = 0;
    int64_t *flat = (int64_t *)malloc(cap * sizeof(int64_t));
    size_t rcap = 64; int nrows = 0;
    size_t *row_start = (size_t *)malloc(rcap * sizeof(size_t));
    int *row_len = (int *)malloc(rcap * sizeof(int));
    if (!flat || !row_start || !row_len) {
        free(flat); free(row_start); free(row_len);
        return ld_fail(LD_ERR_NOMEM, "out of host memory reading the matrix");
    }
    char tok[256];
    int tl = 0, sci = 0, in_row = 0;
    int64_t last = 0;
    size_t cur_start = 0;
    for (size_t p = 0; p <= len; p++) {
        char g = p < len ? text[p] : '\n';
        int end_of_text = (p == len);
        if (!end_of_text && is_entry_char(g)) {
            if (tl < (int)sizeof(tok) - 1) tok[tl++] = g;
            if (g == 'e' || g == 'E') sci = 1;
            continue;
        }
        if (tl > 0) {
            tok[tl] = 0;
            if (sci) {
                double dv;
                if (sscanf(tok, "%le", &dv) == 1) last = (int64_t)dv;
            } else {
                long long v;
                if (sscanf(tok, "%lld", &v) == 1) last = (int64_t)v;
            }
            sci = 0; tl = 0;
            if (n == cap) {
                cap *= 2;
                int64_t *nf = (int64_t *)realloc(flat, cap * sizeof(int64_t));
                if (!nf) { free(flat); free(row_start); free(row_len); return ld_fail(LD_ERR_NOMEM, "out of host memory"); }
                flat = nf;
            }
            if (!in_row) { in_row = 1; cur_start = n; }
            flat[n++] = last;
        }
        if (g == '\n' && in_row) {
            if ((size_t)nrows == rcap) {
                rcap *= 2;
                size_t *ns = (size_t *)realloc(row_start, rcap * sizeof(size_t));
                int *nl = (int *)realloc(row_len, rcap * sizeof(int));
                if (!ns || !nl) { free(ns ? ns : row_start); free(nl ? nl : row_len); free(flat); return ld_fail(LD_ERR_NOMEM, "out of host memory"); }
                row_start = ns; row_len = nl;
            }
            row_start[nrows] = cur_start;
            row_len[nrows] = (int)(n - cur_start);
            nrows++;
            in_row = 0;
        }
    }
    ld_status st = LD_OK;
    int ncols = nrows ? row_len[nrows - 1] : 0;
    if (nrows == 0) st = ld_fail(LD_ERR_INPUT, "the matrix file has no entries");
    for (int i = 0; i < nrows && st == LD_OK; i++)
        if (row_len[i] < ncols)
            st = ld_fail(LD_ERR_INPUT, "row %d has %d entries but the last row has %d", i + 1, row_len[i], ncols);
    int64_t *a = NULL;
    if (st == LD_OK) {
        a = (int64_t *)malloc((size_t)nrows * ncols * sizeof(int64_t));
        if (!a) st = ld_fail(LD_ERR_NOMEM, "out of host memory");
        else for (int i = 0; i < nrows; i++) memcpy(a + (size_t)i * ncols, flat + row_start[i], (size_t)ncols * sizeof(int64_t));
    }
    free(flat); free(row_start); free(row_len);
    if (st != LD_OK) return st;
    *out = a; *rows = nrows; *cols = ncols;
    return LD_OK;
}
