/*
 * Internal declarations shared by the host C code and the CUDA solver.
 */
#ifndef LD_INTERNAL_H
#define LD_INTERNAL_H

#include <stdarg.h>
#include <stddef.h>
#include <stdint.h>

#include "../../../include/lnorms_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define LD_MAX_COLS 4096   /* `length` of the reference (functions.h:2)       */
#define LD_MAX_D 10        /* RANK_OF_NORM (functions.h:3)                    */
#define LD_INDEX_BITS 64   /* NUM_OF_BITS (functions.h:4)                     */

/* Preprocessed problem: the reference's `item` + `item_calc`
 * (functions.h:7-38), plus the stdout text it prints. */
struct ld_problem {
    int R0, C0;            /* as read                                          */
    int64_t *a;            /* R0*C0 working matrix (united lines accumulate)   */
    int d_user;            /* order given on the command line                  */
    char stat;             /* preprocessing flag character                     */
    int marg_user;         /* marginal flag as parsed (d == 1 only)            */
    int *rmark, *cmark;    /* 0 kept; R0 / C0 zero line; +k / -k united (with
                              the same / opposite sign) into line k-1          */
    int R, C;              /* reduced (after transpose)                        */
    int d, marg, transposed, max_rows;
    uint64_t labelings;    /* d^(R-1) (2^(R-1) for d <= 2), saturating          */
    int64_t *red;          /* reduced row-major matrix, fixed row last         */
    const int *orig;       /* markers of the lines the strategy is indexed by  */
    int orig_len;
    char *log;             /* the reference's stdout text so far               */
    size_t log_n, log_cap;
};

void ld_logf(ld_problem *p, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
ld_status ld_fail(ld_status st, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
void ld_clear_error(void);

/* matrix text -> row-major int64 (matrix_read semantics); rows and cols set,
 * *out malloc'ed. */
ld_status ld_parse_matrix_text(const char *text, size_t len, int64_t **out, int *rows, int *cols);

/* preprocessing of a parsed matrix (takes ownership of a) */
ld_status ld_problem_build(int64_t *a, int rows, int cols, int d, char stat, int marginal,
                           ld_problem **out);

/* maximum reduced rows for order d (calc_Parameters, L_CUDA.cu:250-265) */
int ld_max_rows_for(int d);
/* d^(rows-1) (2^(rows-1) for d <= 2), saturating at UINT64_MAX */
uint64_t ld_labelings(int rows, int d);

/* walks [lo, hi) of shard `index` of `count`: equal numbers of walks that
 * pass the label-symmetry test (symmetry.c), tiling [0, d^P) */
ld_status ld_sym_split(int d, int P, int index, int count, uint64_t *lo, uint64_t *hi);
/* completion counts f[(used >> 1)][par][r] (ld_sym_table_len entries): the
 * passing continuations of r more digits after a prefix that has seen the
 * labels in `used` (bit 0 always set) and whose next digit has reflection par */
size_t ld_sym_table_len(int d, int P);
ld_status ld_sym_table(int d, int P, uint64_t *table);

#ifdef __cplusplus
}
#endif
#endif
