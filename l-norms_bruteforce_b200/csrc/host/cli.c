/*
 * The drop-in executable: `L_CUDA number_of_blocks threads_per_block
 * matrix_file d [y|Y|c|C|r|R|other] [m|M]`.
 *
 * Argument checks, their messages and the order of the stdout lines follow
 * arguments_CUDA and main (L_CUDA.cu:361-439); the strategy file follows
 * print_results (functions.h:371-412).  blocks/threads are validated and
 * echoed exactly as the reference does (they set the "num_ofBlock" line),
 * but the kernels pick their own launch shape.  Differences, all on paths
 * where the reference misbehaves: a missing matrix file prints the
 * reference's message and exits with status 255 instead of crashing in
 * fclose(NULL); malformed matrices (no entries, rows shorter than the last)
 * and CUDA failures are reported on stderr with a nonzero exit.
 * LD_VERBOSE=1 adds a timing line on stderr.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ld_internal.h"

int ld_device_max_threads(int device, int *out);   /* solver.cu */

static size_t g_printed;

static void flush_log(const ld_problem *p) {
    const char *s = ld_problem_log(p);
    size_t n = strlen(s);
    if (n > g_printed) { fputs(s + g_printed, stdout); g_printed = n; }
    fflush(stdout);
}

int ld_cli_main(int argc, char **argv) {
    const char *msg = "Use the following command: ./L_CUDA number_of_blocks number_of_threads_per_block filename_of_matrix order_of_the_L_norm";
    int t = 0, sd, blocks, threads, d, marginal;
    char stat;
    g_printed = 0;
    if (argc < 5) {
        printf("Incorrect number of input arguments. %s\n", msg);
        return 255;
    }
    sd = sscanf(argv[1], "%d", &t);
    if (sd == 0 || t < 1) {
        printf("Please make sure that the number of blocks is a positive integer. %s\n", msg);
        return 255;
    }
    blocks = t;
    sd = sscanf(argv[2], "%d", &t);
    if (sd == 0 || t < 1) {
        printf("Please make sure that the number of threads is a positive integer. %s\n", msg);
        return 255;
    }
    threads = t;
    const char *path = argv[3];
    FILE *fp = fopen(path, "r");
    if (fp == NULL) {
        printf("Please make sure that the file containig the matrix exists within this directory. %s\n", msg);
        fflush(stdout);
        return 255;
    }
    fclose(fp);
    sd = sscanf(argv[4], "%d", &t);
    if (sd == 0 || t < 1) {
        printf("Please make sure that the order of the L norm is a positive integer. %s\n", msg);
        return 255;
    }
    d = t;
    stat = argc < 6 ? 'n' : argv[5][0];
    if (argc < 6 || d > 1) marginal = 0;
    else if (argc == 6) marginal = (argv[5][0] == 'm' || argv[5][0] == 'M');
    else marginal = (argv[6][0] == 'm' || argv[6][0] == 'M');
    if (t > LD_MAX_D) {
        printf("The order of the L norm is too large. Please increase the RANK_OF_NORM variable in the code to %d and compile and run it again.\n", t);
        return 255;
    }
    int max_threads = 0;
    if (ld_device_max_threads(0, &max_threads) != 0) {
        fflush(stdout);
        fprintf(stderr, "L_CUDA: no usable CUDA device: %s\n", ld_last_error());
        return 1;
    }
    if (threads > max_threads) {
        printf("The maximum number of threads per block cannot be more than %d.\n", max_threads);
        return 255;
    }

    ld_problem *p = NULL;
    ld_status st = ld_problem_from_file(path, d, stat, marginal, &p);
    if (st != LD_OK) {
        fflush(stdout);
        fprintf(stderr, "L_CUDA: %s\n", ld_last_error());
        return 1;
    }
    flush_log(p);
    st = ld_problem_check_launch(p, blocks, threads);
    flush_log(p);
    if (st != LD_OK) { ld_problem_destroy(p); return 255; }

    ld_result res;
    memset(&res, 0, sizeof res);
    if (p->R == 0) {
        ld_logf(p, "This is a zero matrix.\n");
    } else {
        ld_options opt;
        ld_options_init(&opt);
        st = ld_problem_solve(p, &opt, &res);
        if (st != LD_OK) {
            flush_log(p);
            fprintf(stderr, "L_CUDA: solve failed: %s\n", ld_last_error());
            ld_problem_destroy(p);
            return 1;
        }
    }
    int32_t *strategy = (int32_t *)malloc(sizeof(int32_t) * (size_t)(p->orig_len > 0 ? p->orig_len : 1));
    int32_t count = 0;
    char name[64];
    st = ld_problem_report(p, &res, strategy, p->orig_len, &count, name, sizeof name);
    flush_log(p);
    if (st == LD_OK) {
        FILE *f = fopen(name, "w");
        if (!f) { fprintf(stderr, "L_CUDA: cannot write %s\n", name); st = LD_ERR_IO; }
        else {
            for (int i = 0; i < count; i++) fprintf(f, "%d\n", strategy[i]);
            fclose(f);
        }
    }
    const char *verbose = getenv("LD_VERBOSE");
    if (verbose && verbose[0] == '1')
        fprintf(stderr, "L_CUDA: kernel %d, %d-bit lanes, %llu labelings (%llu evaluated), %.3f ms\n",
                res.kernel_kind, res.lane_bits, (unsigned long long)res.labelings,
                (unsigned long long)res.evaluated, (double)res.kernel_ms);
    free(strategy);
    ld_problem_destroy(p);
    return st == LD_OK ? 0 : 1;
}
