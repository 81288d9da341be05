/* Test infrastructure: the reference's own OpenMP program with its
 * calc_Lnorm (L_OpenMP.c:241-297) replaced by one call into this library.
 *
 * oracle/Makefile (target `binding`) compiles the unmodified L_OpenMP.c,
 * marks its calc_Lnorm weak, and links this file's definition in its place,
 * so the reference's own main, argument handling, parser, preprocessing and
 * print_results (functions.h) run around the library's solve.  This is the
 * stub a maintainer of the reference would write; tests run the result on
 * the golden cases and compare stdout and strategy files byte for byte.
 *
 * The reference's item_calc (functions.h:7-21) arrives after calc_Parameters
 * (L_OpenMP.c:344-376): n is the effective order (after the d reset),
 * mtx_as_vec is the reduced matrix, row-major, with the fixed row (or the
 * marginal row) last -- the layout ld_solve_reduced takes.  The strategy is
 * the rows-1 labels of the reference's Ln_strategy (0/1 for d <= 2, 1 = +1
 * for d = 1; 0..d-1 otherwise), freed by the reference's free_second. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "functions.h"
#include "lnorms_b200.h"

void calc_Lnorm(item_calc* second) {
    const int R = second->iRows_reduced, C = second->iCols_reduced;
    int64_t* a = (int64_t*)malloc(sizeof(int64_t) * (size_t)R * (size_t)C);
    int32_t* lab = (int32_t*)calloc(R > 1 ? (size_t)(R - 1) : 1, sizeof(int32_t));
    second->strategy = (int*)calloc(R > 1 ? (size_t)(R - 1) : 1, sizeof(int));
    if (!a || !lab || !second->strategy) {
        perror("calc_Lnorm");
        exit(-1);
    }
    for (size_t i = 0; i < (size_t)R * (size_t)C; i++) a[i] = second->mtx_as_vec[i];
    ld_result res;
    if (ld_solve_reduced(a, R, C, second->n, second->marginal, NULL, &res, lab) != LD_OK) {
        fprintf(stderr, "%s\n", ld_last_error());
        exit(-1);
    }
    second->Lnorm = (int_type)res.value;
    for (int i = 0; i < R - 1; i++) second->strategy[i] = lab[i];
    free(a);
    free(lab);
}
