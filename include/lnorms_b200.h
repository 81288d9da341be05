/*
 * lnorms_b200.h -- C ABI of the B200-native exact L_d-norm solver.
 *
 * The reference (istvanmarton/L-norms_BruteForce) has no library API: its
 * boundary is the executable `L_CUDA blocks threads matrix d [y|c|r] [m]`
 * (L_CUDA.cu:361-439) built from the stage functions below.  This header
 * exposes one entry point per stage, with plain pointers and sizes only, so
 * a C host (the drop-in CLI in this package, a ctypes/cffi binding, or the
 * reference's own main with its calc_Lnorm body replaced) can call it.
 *
 * Conventions
 *  - Every function returns an ld_status (0 = LD_OK); nothing here exits or
 *    prints.  ld_last_error() gives a one-line message for the calling
 *    thread's last failure.
 *  - The caller owns every host buffer it passes; the library owns device
 *    memory (plans) and host objects it returns (problems), which the caller
 *    releases with the matching *_destroy.
 *  - A plan is single-threaded and runs on one CUDA stream (its own, or the
 *    one given in ld_options).
 *  - Matrix entries are int64 on the host.  The device path computes in
 *    packed int8x4, int32 or int64 lanes, chosen from an exact bound on
 *    every partial column sum, so results never overflow.
 */
#ifndef LNORMS_B200_H
#define LNORMS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    LD_OK = 0,
    LD_ERR_ARG = 1,      /* invalid argument                                    */
    LD_ERR_INPUT = 2,    /* malformed matrix text (no entries, ragged rows)     */
    LD_ERR_LIMIT = 3,    /* too many rows for the Gray index, or > 4096 columns */
    LD_ERR_CUDA = 4,     /* a CUDA runtime call failed                          */
    LD_ERR_NODEV = 5,    /* no CUDA device (the library has no CPU fallback)    */
    LD_ERR_IO = 6,       /* file could not be opened                            */
    LD_ERR_TIMEOUT = 7,  /* a bounded device-side wait gave up                  */
    LD_ERR_NOMEM = 8     /* host allocation failed                              */
} ld_status;

/* Result of one solve. */
typedef struct {
    int64_t value;         /* the L_d norm (LM for marginal problems)                */
    uint64_t gray_index;   /* smallest Gray-code index attaining it (tie-break of
                              L_CUDA.cu:80 strict '>' and :347 strict '<')          */
    uint64_t labelings;    /* labelings the solve covered (evaluated, or skipped by
                              a bound or by label symmetry)                        */
    float kernel_ms;       /* device time of the solve's launches (CUDA events)     */
    int32_t kernel_kind;   /* LD_KERNEL_* actually used                             */
    int32_t lane_bits;     /* 8, 16, 32 or 64: arithmetic lane width used           */
    uint64_t h2d_bytes;    /* host-to-device bytes this solve copied                */
    uint64_t d2h_bytes;    /* device-to-host bytes this solve copied                */
    uint64_t evaluated;    /* labelings the kernels computed a value for (fewer
                              than `labelings` when walks were skipped by label
                              symmetry or by a bound)                              */
} ld_result;

enum {
    LD_KERNEL_NONE = 0,     /* zero matrix: nothing launched                     */
    LD_KERNEL_TABLE = 1,    /* register kernel with a shared-memory table of the
                               low rows' partial sums (d = 1, LM, 2, 3)           */
    LD_KERNEL_WIDE = 2      /* column-parallel kernel (any d <= 10, <= 4096 cols,
                               int32 or int64)                                    */
};

/* Tuning and placement knobs; ld_options_init() fills the defaults (0/-1 =
 * automatic).  None of them changes the result. */
typedef struct {
    int32_t device;             /* CUDA device ordinal                            */
    int32_t low_rows;           /* rows tabulated in shared memory (-1 auto)      */
    int32_t threads_per_block;  /* 0 auto                                         */
    int32_t blocks;             /* 0 auto (a multiple of the SM count)            */
    int32_t tile;               /* prefixes walked together per thread (0 auto)   */
    int32_t kernel;             /* 0 auto, else LD_KERNEL_TABLE / LD_KERNEL_WIDE  */
    int32_t lane_bits;          /* 0 auto, else force 16 / 32 / 64 (>= needed)    */
    int32_t shard_index;        /* this device's part of a solve split over       */
    int32_t shard_count;        /* shard_count devices (0 or 1: the whole range)  */
    int32_t prune_policy;       /* ld_solve_pruned: 0 = run the plain enumeration
                                   instead when more than a quarter of the walk
                                   prefixes survive their bound; 1 = always scan */
    int32_t enumerate_all;      /* d >= 3: 0 = skip walks that hold no smallest
                                   index of a label-permutation class (see
                                   ld_symmetry_walks); 1 = evaluate every walk   */
    int32_t batch_split;        /* ld_batch_create, int32 classes of 40..64 words:
                                   0 = the autotuner picks the column-split or
                                   the plain instance (plain when not tuned);
                                   1 = always column-split; -1 = never          */
    int32_t column_split;       /* table kernel, one solve: lanes that share one
                                   high index, each holding a slice of the
                                   columns.  0 = only when the matrix is too
                                   wide for one thread's registers (d <= 3:
                                   > 64 int32 / > 128 8-bit columns; d >= 4:
                                   > 16 / > 32); 2, 4 or 8 = that many lanes
                                   whenever an instance fits; -1 = never (the
                                   wide kernel takes wide matrices)            */
    int32_t paired_walks;       /* table kernel, d <= 3: 0 = two high indices per
                                   thread against each table read when every
                                   thread has at least two walks; -1 = one   */
    int32_t pack16;             /* table kernel: 0 = keep two running maxima in
                                   one word (16 bits each) when every value is
                                   below 65536; -1 = one maximum per word    */
    int32_t walk_fetch;         /* table kernel: 0 = warps fetch walks from a
                                   counter as they finish (balanced); -1 =
                                   every thread takes a fixed share         */
    int32_t batch_row_search;   /* ld_batch_create with autotune: 1 = also try
                                   one or two low rows fewer per int32 class
                                   (measured: no faster replay on the 4096-
                                   matrix batch, 4x the creation time); 0 = the
                                   largest table that fits                   */
    void *stream;               /* cudaStream_t, NULL = the plan's own stream      */
} ld_options;

void ld_options_init(ld_options *opt);

/* ---------------------------------------------------------------------- */
/* Stage 1+2: read and preprocess.                                          */
/* Replaces matrix_read (functions.h:40-79) and load_parameters             */
/* (L_CUDA.cu:414-423: eliminate_zero_rows_cols functions.h:109-151,         */
/* calc_reduce_matrix_rows :237-262, calc_reduce_matrix_cols :264-289,       */
/* calc_reduce_matrix_cols_sign :193-235, delete_rows/cols :153-191,         */
/* convert_mtx_to_vec :291-329) and the d reset of calc_Parameters           */
/* (L_CUDA.cu:244-248).  `stat` is the preprocessing flag character          */
/* (y/Y/r/R/c/C, anything else = none); `marginal` is honoured for d == 1    */
/* only, as arguments_CUDA does (L_CUDA.cu:401).  The problem keeps the      */
/* lines the reference prints on stdout; see ld_problem_log.                 */
typedef struct ld_problem ld_problem;

ld_status ld_problem_from_text(const char *text, size_t len, int32_t d, char stat,
                               int32_t marginal, ld_problem **out);
ld_status ld_problem_from_file(const char *path, int32_t d, char stat, int32_t marginal,
                               ld_problem **out);
/* Row-major rows x cols entries, as if read from a file. */
ld_status ld_problem_from_matrix(const int64_t *a, int32_t rows, int32_t cols, int32_t d,
                                 char stat, int32_t marginal, ld_problem **out);
void ld_problem_destroy(ld_problem *p);

/* Reduced shape: rows/cols after preprocessing (and transpose), effective d,
 * marginal actually used, and the number of labelings (0 for a zero matrix;
 * saturates at UINT64_MAX). */
typedef struct {
    int32_t rows_in, cols_in;
    int32_t rows, cols;
    int32_t d_user, d;
    int32_t marginal_user, marginal;
    int32_t transposed;
    int32_t max_rows;          /* maximum length of the strategy vector          */
    uint64_t labelings;
} ld_problem_info;
ld_status ld_problem_get_info(const ld_problem *p, ld_problem_info *info);
/* The reduced matrix handed to the solver (mtx_as_vec of the reference):
 * rows*cols int64, row-major, fixed (or marginal) row last. */
ld_status ld_problem_reduced(const ld_problem *p, int64_t *out, size_t cap);
/* Text the reference prints up to this stage (NUL-terminated, owned by p). */
const char *ld_problem_log(const ld_problem *p);

/* calc_Parameters' launch clamp and limit checks (L_CUDA.cu:267-278):
 * appends "num_ofBlock ..." and "maximum length ..." to the log; returns
 * LD_ERR_LIMIT (with the reference's message appended) when the reduced
 * matrix exceeds its row or column limit. */
ld_status ld_problem_check_launch(ld_problem *p, int32_t blocks, int32_t threads);

/* ---------------------------------------------------------------------- */
/* Stage 3: solve.  Replaces calc_Lnorm (L_CUDA.cu:281-359): device upload, */
/* the L1/LM/L2/L3/Ln kernels (L_CUDA.cu:14-240) and the host argmax         */
/* (L_CUDA.cu:341-348).  A zero matrix (rows == 0) yields value 0 without a  */
/* launch, as main does (L_CUDA.cu:432).                                     */
ld_status ld_problem_solve(ld_problem *p, const ld_options *opt, ld_result *res);

/* Same, for an already reduced matrix (mtx_as_vec layout: row-major, the
 * last row carries the fixed label / the marginal row).  d is the effective
 * order.  `strategy` (may be NULL) receives rows-1 labels: 0/1 for d <= 2
 * (1 = +1 for d == 1), 0..d-1 otherwise -- second->strategy of the
 * reference. */
ld_status ld_solve_reduced(const int64_t *mtx_as_vec, int32_t rows, int32_t cols, int32_t d,
                           int32_t marginal, const ld_options *opt, ld_result *res,
                           int32_t *strategy);

/* No counterpart in the reference.  The same solve as ld_solve_reduced for
 * callers that must not allocate GPU memory (cudaMalloc/cudaFree can
 * synchronize the device, and fail once another framework in the process
 * holds nearly all of its memory): all device working memory is one 64 KiB
 * file-scope __device__ array, reserved on every GPU that loads the library.
 * Host matrix in, host result out.  `stream` NULL means the legacy default
 * stream, which synchronises with every blocking stream of the device; pass
 * a cudaStreamNonBlocking stream to keep other work running.  Each call
 * waits for its stream before returning.  Limits: d <= 3, <= 63 rows,
 * <= 64 columns (<= 128 when every partial column sum fits in 8 bits),
 * column sums within 32 bits; larger inputs get LD_ERR_LIMIT.  At d = 3 it
 * skips the same label-permuted walks as ld_solve_reduced.  The first call
 * on a device looks up the array's address (make it before any stream
 * capture on that device).  Calls share the array and are serialised by a
 * host lock; GPU work of two calls must not overlap.  kernel_ms is 0. */
ld_status ld_solve_reduced_noalloc(const int64_t *mtx_as_vec, int32_t rows, int32_t cols,
                                   int32_t d, int32_t marginal, int32_t device, void *stream,
                                   ld_result *res, int32_t *strategy);

/* ---------------------------------------------------------------------- */
/* Pruned exact search (no counterpart in the reference: it speeds the      */
/* enumeration of calc_Lnorm up without changing its answer).  Blocks of    */
/* labelings whose exact integer upper bound (|prefix column sums| + the    */
/* norm of the remaining rows, per message) is below the incumbent are      */
/* skipped; ties are never skipped, so value and Gray index equal           */
/* ld_solve_reduced's.  `incumbent_labels` (rows-1 labels, may be NULL) is  */
/* a labeling whose value the host recomputes.  d <= 3 inside the table     */
/* kernel's range; other inputs fall back to the plain enumeration          */
/* (stats->pruned = 0).                                                     */
typedef struct {
    uint64_t walks_total, walks_kept;         /* top-row prefixes, and those not pruned */
    uint64_t highs_total, highs_visited, highs_kept;  /* high indices (blocks of `block` labelings) */
    uint64_t block;                           /* labelings per high index                */
    int64_t incumbent;                        /* value of the incumbent (INT64_MIN: none) */
    float bound_ms, scan_ms;                  /* device time of the two launches          */
    int32_t pruned;                           /* 1: pruned kernels ran; 0: plain fallback */
    int32_t low_rows, walk_rows;              /* rows tabulated / walked per prefix       */
} ld_prune_stats;
ld_status ld_solve_pruned(const int64_t *mtx_as_vec, int32_t rows, int32_t cols, int32_t d,
                          int32_t marginal, const ld_options *opt, const int32_t *incumbent_labels,
                          ld_result *res, int32_t *strategy, ld_prune_stats *stats);

/* Single-row-move local search on the GPU (no counterpart in the reference):
 * n starting labelings (n x (rows-1) labels) are improved by steepest-ascent
 * moves of one row's label until no move gains (or max_rounds, 0 = 4*rows);
 * values[n] and labels[n x (rows-1)] receive the results.  d <= 3,
 * <= 64 rows, <= 128 columns. */
ld_status ld_local_search(const int64_t *mtx_as_vec, int32_t rows, int32_t cols, int32_t d,
                          int32_t marginal, const int32_t *starts, int32_t n, int32_t max_rounds,
                          int32_t device, int64_t *values, int32_t *labels);

/* Labels of rows 0..rows-2 for a Gray index (the BRGC word of L_CUDA.cu:61-63,
 * the d-ary reflected word of L_CUDA.cu:204-206). */
ld_status ld_gray_labels(uint64_t index, int32_t rows, int32_t d, int32_t *labels);

/* ---------------------------------------------------------------------- */
/* Stage 4: output.  Replaces print_results (functions.h:371-412): the       */
/* "L%d is: %d" / "LM is: %d" line is appended to the log, and `strategy`    */
/* (capacity cap) receives one label per ORIGINAL row (column if the matrix  */
/* was transposed) in the file's encoding (+-1 for d == 1, 0..d-1 else);      */
/* *count gets the number written; name gets "strategy_L%d.txt" or          */
/* "strategy_LM.txt". */
ld_status ld_problem_report(ld_problem *p, const ld_result *res, int32_t *strategy,
                            int32_t cap, int32_t *count, char *name, size_t name_cap);

/* ---------------------------------------------------------------------- */
/* Plans: a device-resident reduced matrix for repeated solves (bench and   */
/* batch callers).  Same arguments as ld_solve_reduced.                      */
typedef struct ld_plan ld_plan;
ld_status ld_plan_create(const int64_t *mtx_as_vec, int32_t rows, int32_t cols, int32_t d,
                         int32_t marginal, const ld_options *opt, ld_plan **out);
/* Enqueue one full solve on the plan's stream; no host synchronisation. */
ld_status ld_plan_launch(ld_plan *plan);
/* Wait for the last launch and read its 16-byte result. */
ld_status ld_plan_result(ld_plan *plan, ld_result *res, int32_t *strategy);
/* Gray-index range [lo, hi) the plan enumerates (its shard, or everything).
 * Shards of the same problem on identical devices tile [0, labelings). */
ld_status ld_plan_range(const ld_plan *plan, uint64_t *lo, uint64_t *hi);
/* One-line description of the kernel configuration the plan chose. */
ld_status ld_plan_describe(const ld_plan *plan, char *buf, size_t cap);
/* The stream the plan launches on (cudaStream_t). */
void *ld_plan_stream(const ld_plan *plan);
/* Device address of the plan's 16-byte result {int64 value; uint64 index},
 * valid after a launch completes on the plan's stream (for callers that
 * combine shards on the device, e.g. with an NCCL all-reduce). */
void *ld_plan_result_device(const ld_plan *plan);
void ld_plan_destroy(ld_plan *plan);

/* ---------------------------------------------------------------------- */
/* Batched solves (no counterpart in the reference: it runs one matrix per   */
/* process).  `count` reduced matrices (mtx_as_vec layout, mats[p] with      */
/* rows[p] x cols[p] entries, order ds[p], marginal flags margs[p] or NULL)  */
/* are solved together: per lane class one persistent kernel pulls          */
/* (matrix, walk range) chunks from a device work queue; the class kernels   */
/* run concurrently and, with the per-matrix fold and the result copy, are   */
/* captured in one CUDA graph at creation.  Matrices outside the classes     */
/* (d >= 4, wider, 64-bit sums) get their own plans inside the same graph.   */
/* autotune != 0 times chunk size and grid size per class on the class's     */
/* largest matrices (cached per class shape for the process).  Results are   */
/* the ones ld_solve_reduced gives for each matrix.                          */
typedef struct ld_batch ld_batch;
ld_status ld_batch_create(int32_t count, const int64_t *const *mats, const int32_t *rows,
                          const int32_t *cols, const int32_t *ds, const int32_t *margs,
                          const ld_options *opt, int32_t autotune, ld_batch **out);
/* Replay the graph on the batch's stream (no host synchronisation). */
ld_status ld_batch_launch(ld_batch *b);
/* Wait for the last launch; values[count], gray_indices[count] (may be NULL),
 * *ms = device time of the launch (may be NULL). */
ld_status ld_batch_results(ld_batch *b, int64_t *values, uint64_t *gray_indices, float *ms);
ld_status ld_batch_describe(const ld_batch *b, char *buf, size_t cap);
/* evaluated[count]: labelings the kernels compute a value for, per matrix
 * (below the matrix's labelings where label symmetry skips walks). */
ld_status ld_batch_evaluated(const ld_batch *b, uint64_t *evaluated);
void ld_batch_destroy(ld_batch *b);

/* ---------------------------------------------------------------------- */
/* Proposal network for the pruned search (no counterpart in the reference): */
/* a 44 -> 256 -> 256 -> 44 ReLU perceptron whose GEMMs run on the tensor    */
/* cores (bf16 operands, fp32 accumulation, tcgen05 + TMEM), trained with    */
/* Adam on fp32 master weights against masked binary cross-entropy.  Rows   */
/* of x are 44 features, rows of t / mask 44 targets in [0,1] and weights   */
/* (0 drops an entry).  Parameters travel as one flat fp32 array: W1[256x44] */
/* b1[256] W2[256x256] b2[256] W3[44x256] b3[44] (ld_mlp_param_count()).    */
/* A network object owns its device buffers, pinned staging, stream and two
 * captured CUDA graphs (a training step, a forward pass); use it from one
 * thread at a time. */
typedef struct ld_mlp ld_mlp;
/* batch: rows per device pass, a positive multiple of 128.  skip: weight of
 * a parameter-free residual path, logits = W3 h2 + b3 + skip * x (the
 * input and output widths are equal; 0 turns it off). */
ld_status ld_mlp_create(int32_t batch, uint64_t seed, float skip, int32_t device, ld_mlp **out);
int64_t ld_mlp_param_count(void);
ld_status ld_mlp_get_params(ld_mlp *net, float *params);
ld_status ld_mlp_set_params(ld_mlp *net, const float *params);
/* logits[rows x 44] for x[rows x 44]; any number of rows. */
ld_status ld_mlp_forward(ld_mlp *net, const float *x, int32_t rows, float *logits);
/* Gradients of the mean masked loss (flat parameter layout; grads or loss
 * may be NULL) for rows <= batch, no update. */
ld_status ld_mlp_gradients(ld_mlp *net, const float *x, const float *t, const float *mask,
                           int32_t rows, float *grads, float *loss);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on rows <= batch. */
ld_status ld_mlp_train_step(ld_mlp *net, const float *x, const float *t, const float *mask,
                            int32_t rows, float lr, float *loss);
void ld_mlp_destroy(ld_mlp *net);
/* The tensor-core GEMM alone, for tests: C[M x N] (fp32) = A[M x K] *      */
/* B[N x K]^T with A, B given as bf16 bit patterns; M % 128 == 0,           */
/* N % 64 == 0, K % 64 == 0. */
ld_status ld_tc_gemm(const uint16_t *A, const uint16_t *B, int32_t M, int32_t N, int32_t K,
                     float *C, int32_t device);

/* ---------------------------------------------------------------------- */
/* The drop-in executable: `blocks threads matrix d [y|c|r] [m]`, same      */
/* argument checks, stdout lines and strategy file as L_CUDA's main and     */
/* arguments_CUDA (L_CUDA.cu:361-439).  Returns the process exit status.    */
int ld_cli_main(int argc, char **argv);

/* ---------------------------------------------------------------------- */
/* Resumable solves (no counterpart in the reference).  The solve runs as   */
/* `pieces` shards (ld_options.shard_index / shard_count semantics: equal    */
/* work per piece) one after another on one device; after each piece the    */
/* next piece, the Gray range covered and the best (value, index) so far    */
/* are written to `checkpoint_path` (a small text file, replaced            */
/* atomically).  A later call with the same matrix, d, marginal, pieces and */
/* enumerate_all continues after the last recorded piece; a checkpoint of   */
/* another problem is refused (LD_ERR_ARG), and so is a piece that would    */
/* not start where the recorded coverage ends (changed options or device).  */
/* At most max_pieces pieces run per call (<= 0: all).  *done = 1 once every */
/* piece has run; res (and strategy, rows-1 labels) then hold what          */
/* ld_solve_reduced gives, with labelings / evaluated / kernel_ms summed    */
/* over the pieces.  Before that res holds the best so far.                 */
ld_status ld_solve_resumable(const int64_t *a, int32_t rows, int32_t cols, int32_t d, int32_t marginal,
                             const ld_options *opt, int32_t pieces, const char *checkpoint_path,
                             int32_t max_pieces, int32_t *done, ld_result *res, int32_t *strategy);

/* ---------------------------------------------------------------------- */
/* Label symmetry (d >= 3; the reference enumerates every labeling,         */
/* L_CUDA.cu:186-240).  The fixed row has label 0 and the value is          */
/* unchanged when labels 1..d-1 are permuted, so the smallest Gray index     */
/* attaining the maximum is the smallest index of its class.  A walk (the   */
/* table kernel's block of high indices, the wide kernel's run of d^L       */
/* consecutive indices) fixes the top `prefix_digits` base-d digits of the  */
/* index: the walk number w.  A walk whose prefix cannot begin a class      */
/* minimum is skipped by the table and wide kernels, the batch's d = 3      */
/* class and the pruned search's walk bound (ld_options.enumerate_all = 0). */
/* For d <= 2 every walk passes.                                             */
/* 1 when walk w passes the class-minimum test, else 0. */
int32_t ld_symmetry_walk_ok(int32_t d, int32_t prefix_digits, uint64_t w);
/* Walks in [lo, hi) that pass (hi <= d^prefix_digits). */
ld_status ld_symmetry_walks(int32_t d, int32_t prefix_digits, uint64_t lo, uint64_t hi, uint64_t *count);
/* *w = the passing walk of the given rank (0-based, increasing walk numbers);
 * the table and wide kernels hand out walks by rank. */
ld_status ld_symmetry_walk_at(int32_t d, int32_t prefix_digits, uint64_t rank, uint64_t *w);

/* ---------------------------------------------------------------------- */
/* Spectral basis for the learned search's proposals (no counterpart in the */
/* reference): out (cols x k, row-major) = the k leading eigenvectors of    */
/* A^T A, each with its largest-magnitude component positive, by subspace   */
/* iteration with a Rayleigh-Ritz step (cols <= 64, k <= 8; columns beyond  */
/* cols are zero).  *iterations (may be NULL) gets the iterations used.     */
ld_status ld_spectral_basis(const int64_t *a, int32_t rows, int32_t cols, int32_t k, double *out,
                            int32_t *iterations);

/* ---------------------------------------------------------------------- */
/* Strategy verifier (no counterpart in the reference).  The value, on the   */
/* matrix as read, of the labeling a strategy file records (the file of     */
/* print_results, functions.h:371-412: one entry per input row, or per      */
/* column when the d = 1 problem was transposed; +1/-1 for d = 1, 0..d-1    */
/* otherwise).  `text`, d, stat and marginal as for ld_problem_from_text.   */
ld_status ld_strategy_value(const char *text, size_t len, int32_t d, char stat, int32_t marginal,
                            const int32_t *strategy, int32_t count, int64_t *value);
/* `L_verify matrix_file strategy_file d [y|c|r] [m]`: prints the solver's   */
/* value line ("L3 is: 258") for the strategy; returns the exit status.     */
int ld_verify_main(int argc, char **argv);

/* Integer roofline denominator: sustained 32-bit integer ALU operations per
 * second of the device, from a microbenchmark of independent add/xor
 * dependency chains (no counterpart in the reference).  *ms gets the
 * fastest launch time. */
ld_status ld_measure_int32_peak(int32_t device, double *ops_per_second, double *ms);

/* Last error message of the calling thread ("" if none). */
const char *ld_last_error(void);
/* Library version string. */
const char *ld_version(void);

#ifdef __cplusplus
}
#endif
#endif /* LNORMS_B200_H */
