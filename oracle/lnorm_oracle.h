/*
 * lnorm_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C CPU restatement of the brute-force L_d-norm solver of
 * istvanmarton/L-norms_BruteForce (functions.h, L_OpenMP.c, L_CUDA.cu).
 * It is the checker for the product's CUDA path: only tests/, the smoke
 * check and bench.py's CPU-baseline leg may load it.  The product library
 * never links or calls anything in this directory.
 *
 * Arithmetic is int64 throughout (the reference uses int, which overflows
 * for large entries; inside the int range the results are identical).
 * Parity of this restatement is pinned against outputs of the reference's
 * own L_OpenMP.c, built from its sources by oracle/Makefile into
 * oracle/_ref/, on the fixtures in tests/golden/.
 */
#ifndef LNORM_ORACLE_H
#define LNORM_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Full CLI pipeline of the CUDA drop-in (L_CUDA.cu:425-439 main):
 * parse `text` (the matrix file's bytes), preprocess, enumerate, and
 * produce the exact stdout text and strategy-file text the reference
 * prints.  blocks/threads are the CLI's launch arguments (they only change
 * the "num_ofBlock" line).  Returns 0 on success, -1 when the reference
 * would exit(-1) (stdout then holds the lines printed before the exit),
 * -2 on malformed input the reference treats as undefined behaviour.
 * value_out receives the norm; strategy_name receives "strategy_L3.txt" etc. */
int or_run_cli(const char *text, size_t len, int blocks, int threads, int d,
               char stat, int marginal, int nthreads,
               char *out_stdout, size_t cap_stdout,
               char *out_strategy, size_t cap_strategy,
               char *strategy_name, size_t cap_name, int64_t *value_out);

/* Preprocessing only (functions.h:40-329 + calc_Parameters' d-reset):
 * writes the reduced row-major matrix (rows*cols entries; last row is the
 * fixed row, marginal row swapped there) into red (capacity cap entries).
 * Returns 0, or -1 on an exit path, -2 on malformed input. */
int or_preprocess(const char *text, size_t len, int d, char stat, int marginal,
                  int64_t *red, size_t cap, int *rows, int *cols,
                  int *d_eff, int *marginal_eff, int *transposed);

/* Exhaustive enumeration of the reduced matrix (L_OpenMP.c:15-239):
 * max value over all labelings with the last row fixed, and the smallest
 * Gray index attaining it.  Gray indices in [lo, hi) only (hi = 0 means
 * the full range).  nthreads OpenMP threads split the range. */
int or_enumerate(const int64_t *a, int rows, int cols, int d, int marginal,
                 uint64_t lo, uint64_t hi, int nthreads,
                 int64_t *value, uint64_t *index);

/* Number of labelings: 2^(rows-1) for d<=2, d^(rows-1) for d>=3. */
uint64_t or_total(int rows, int d);

/* Labels of rows 0..rows-2 for Gray index N (functions.h:350-369 tables,
 * L_CUDA.cu:61-63 / 204-206 seeds): 0/1 for d<=2, 0..d-1 otherwise. */
void or_labels(uint64_t N, int rows, int d, int32_t *labels);

/* Value of one labeling (labels of rows 0..rows-2; the last row has
 * label 1 (+1) for d==1 and 0 for d>=2). */
int64_t or_value(const int64_t *a, int rows, int cols, int d, int marginal,
                 const int32_t *labels);

#ifdef __cplusplus
}
#endif
#endif
