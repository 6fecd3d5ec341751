/*
 * specspars.h -- C ABI of the B200-native spec_spars sparsification path.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, returns an
 * int status (SSP_OK == 0) and never throws across the boundary.  The message
 * of the last failure on the calling thread is available from
 * ssp_last_error().
 *
 * Reference interfaces replaced (tenchd/spec_spars):
 *   ssp_run_solve_lap   <- ffi::run_solve_lap          src/lib.rs:103, include/example.h:18,
 *                                                      src/example.cc:668-703
 *   ssp_solve_lap       <- same, with explicit options/report and host or device buffers
 *   ssp_sparsify        <- Sparsifier::sparsify         src/sparsifier.rs:722-770, driven like
 *                          InputStream::run_stream      src/stream.rs:40-64
 *   ssp_sparsify_mtx    <- sparsify_dataset             src/lib.rs:145-166 (read .mtx, sparsify, write .mtx)
 *   ssp_sparsify_laplacian <- a Laplacian input, as Sparsifier::from_matrix loads one  src/sparsifier.rs:299-300
 *   ssp_params_default  <- SparsifierParameters::new_default  src/sparsifier.rs:182-209
 *   ssp_params_new      <- SparsifierParameters::new          src/sparsifier.rs:163-179
 *   ssp_params_cli      <- the knobs sparsify_dataset hard-codes, src/lib.rs:149-156
 *   ssp_read_mtx / ssp_write_mtx <- utils::read_mtx / write_mtx  src/utils.rs:149-154,189-191
 *   stage entry points (ssp_stage_*) expose each kernel of the path for parity testing:
 *     edges+Laplacian <- Triplet::insert/to_csc, form_laplacian  src/sparsifier.rs:48-87,693-709
 *     sketch          <- jl_sketch_colwise_flat                  src/sparsifier.rs:490-539
 *     factor          <- factorization_driver                    src/example.cc:332-471
 *     diff norms      <- compute_diff_norms                      src/sparsifier.rs:565-583
 *     probabilities   <- compute_probs                           src/sparsifier.rs:542-562
 *     sample/apply    <- sample_and_reweight + apply_reweightings src/sparsifier.rs:625-691
 */
#ifndef SPECSPARS_H
#define SPECSPARS_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define SSP_OK 0
#define SSP_ERR_INVALID (-1)       /* malformed input / bad argument */
#define SSP_ERR_CUDA (-2)          /* CUDA runtime failure */
#define SSP_ERR_NOMEM (-3)         /* device or host allocation failed */
#define SSP_ERR_NOT_CONVERGED (-4) /* PCG relative residual >= 0.01 (reference throws, example.cc:566) */
#define SSP_ERR_CAPACITY (-5)      /* internal pool capacity exceeded */
#define SSP_ERR_IO (-6)            /* file I/O or .mtx parse error */
#define SSP_ERR_NO_DEVICE (-7)     /* no CUDA device visible */
#define SSP_ERR_PENDING (-8)       /* ssp_poll / ssp_wait: the request has not finished yet */

#define SSP_MEM_HOST 0
#define SSP_MEM_DEVICE 1

/* JL dimension rule */
#define SSP_JL_DIM_REF 0  /* k = ceil(log2(n) * jl_factor)   (sparsifier.rs:272) */
#define SSP_JL_DIM_24 1   /* k = ceil(24 ln(n) / eps^2)                           */
/* sketch entry scale */
#define SSP_JL_SCALE_FIXED 0      /* entries +-jl_scaling_factor (lib.rs:151)   */
#define SSP_JL_SCALE_INV_SQRT_K 1 /* entries +-1/sqrt(k)                        */
/* arithmetic of the PCG solve */
#define SSP_PRECISION_FP64 0  /* every vector and matrix in FP64                                     */
#define SSP_PRECISION_MIXED 1 /* SpMM, triangular solves and vectors in FP32 with FP64 dot products,
                                 inside FP64 iterative refinement to the same tolerance                */
#define SSP_PRECISION_PC32 2  /* FP64 PCG (vectors, SpMM, dot products) whose preconditioner runs in FP32:
                                 the triangular solves read FP32 factor values and gather FP32 rows    */
/* where the preconditioner's level-launch shapes came from (ssp_stats.trsv_shapes) */
#define SSP_TRSV_RULE 0     /* fixed rule: levels of at most 1024 rows 8 columns per warp row, wider ones 32 */
#define SSP_TRSV_TUNED 1    /* measured in this call: the solve's first applications, one per width, timed
                               level by level; the fastest width per level kept                          */
#define SSP_TRSV_CACHED 2   /* measured by an earlier call on the same factor shape (context cache)        */
#define SSP_TRSV_FORCED 3   /* one width for every level, from the environment (SSP_TRSV_WIDTH)            */
/* reweighting of kept edges */
#define SSP_REWEIGHT_INV_SQRT_P 0 /* w / sqrt(p)  (sparsifier.rs:657)           */
#define SSP_REWEIGHT_INV_P 1      /* w / p        (stream_sparsify.jl:135)      */

typedef struct ssp_context ssp_context;

/* Sparse matrix in compressed-sparse-column form (for the symmetric matrices
 * of this path CSC == CSR).  Row indices strictly increasing within a column. */
typedef struct {
    int64_t n;               /* square: n x n */
    int64_t nnz;
    const int64_t* colptr;   /* [n+1] */
    const int32_t* rowidx;   /* [nnz] */
    const double* values;    /* [nnz] */
    int32_t mem;             /* SSP_MEM_HOST or SSP_MEM_DEVICE */
} ssp_csc;

/* Library-allocated CSC result; release with ssp_csc_free(). */
typedef struct {
    int64_t n;
    int64_t nnz;
    int64_t* colptr;
    int32_t* rowidx;
    double* values;
    int32_t mem;             /* where the arrays live */
    int32_t owned_by_context;/* device results may live in the context until its next call */
} ssp_csc_out;

/* SparsifierParameters (sparsifier.rs:146-159) plus the options this build adds. */
typedef struct {
    double epsilon;
    int32_t beta_constant;
    int32_t row_constant;
    int32_t verbose;
    double jl_factor;
    double jl_scaling_factor;
    uint64_t sketch_seed;
    uint64_t sampling_seed;
    int32_t bench;
    int32_t sketch_uniform;
    int32_t streaming;       /* accepted, not acted on: the reference's CLI path sets it false (lib.rs:155) */
    const char* output_file; /* "" or NULL: do not write */
    /* additions */
    int32_t jl_dim_rule;     /* SSP_JL_DIM_* */
    int32_t jl_scale_rule;   /* SSP_JL_SCALE_* */
    int32_t prob_variance_correction; /* 1: divide probabilities by k*s^2 instead of k */
    int32_t reweight;        /* SSP_REWEIGHT_* */
    double pcg_tol;          /* relative residual stop */
    double pcg_abs_tol;      /* absolute residual stop (reference: sqrt(2e-7), custom_cg.hpp:159,213) */
    int32_t pcg_max_iters;   /* reference: 400 (custom_cg.hpp:153) */
    uint64_t factor_seed;    /* elimination order + fill sampling */
    int64_t dense_threshold; /* live-vertex count that switches elimination to the dense tail */
    int64_t factor_max_degree; /* stop eliminating once the Schur complement's average degree exceeds
                                  this; the rest is preconditioned by its diagonal (0 = eliminate all,
                                  -1 = choose by the autotuner) */
    int32_t jl_dim_override;   /* > 0: use exactly this many JL columns instead of jl_dim_rule */
    int32_t precision;         /* SSP_PRECISION_* of the PCG solve */
} ssp_params;

typedef struct {
    int64_t n;
    int64_t m_in;            /* edges before (sparsifier.rs:686) */
    int64_t m_out;           /* edges after  (sparsifier.rs:688) */
    int32_t k;               /* JL columns */
    double beta;
    int64_t nnz_factor;
    int32_t factor_levels;
    int32_t pcg_max_iters_used;
    double pcg_mean_iters;
    double pcg_max_relres;
    /* per-stage milliseconds (Benchmarker phases, utils.rs:126-143) */
    double ms_assembly, ms_sketch, ms_factor, ms_solve, ms_leverage, ms_sample, ms_total;
    int64_t kernels_launched;
    /* device time of the PCG's Laplacian products and preconditioner applications (CUDA events) */
    double ms_spmm;
    int64_t n_spmm;
    double ms_precond;
    int64_t n_precond;
    int64_t nnz_laplacian;
    int64_t factor_max_degree_used; /* truncation actually used (autotuner's choice when requested) */
    double ms_autotune;             /* device time spent choosing it (included in ms_factor) */
    int32_t pcg_refinements;        /* SSP_PRECISION_MIXED: FP64 refinement rounds (0 in FP64 mode) */
    int32_t pcg_fp64_rounds;        /* ... of which ran an FP64 inner solve after FP32 stopped contracting */
    int32_t spmm_slabs;             /* column slabs of the PCG's Laplacian product (1 = one pass) */
    int32_t trsv_shapes;            /* SSP_TRSV_*: how the preconditioner's level-launch shapes were chosen */
    int32_t trsv_levels_w8;         /* level launches (forward + backward) at 8 columns per warp row, */
    int32_t trsv_levels_w16;        /* ... at 16, */
    int32_t trsv_levels_w32;        /* ... at 32 (runs of thin levels are not counted: always 8) */
    double ms_trsv_tune;            /* device time of the applications that measured them (real
                                       applications of the solve; 0 when taken from the cache) */
} ssp_stats;

typedef struct {
    double tol;
    double abs_tol;
    int32_t max_iters;
    uint64_t factor_seed;
    int64_t dense_threshold;
    int32_t verbose;
    int64_t factor_max_degree;
    int32_t precision;       /* SSP_PRECISION_* */
} ssp_solve_opts;

typedef struct {
    int32_t k;
    int32_t max_iters_used;
    double mean_iters;
    double max_relres;
    int32_t not_converged;
    int64_t nnz_factor;
    int32_t factor_levels;
    double ms_factor;
    double ms_solve;
    int64_t factor_max_degree_used;
    int32_t refinements;     /* SSP_PRECISION_MIXED: FP64 refinement rounds */
    int32_t fp64_rounds;
    int32_t spmm_slabs;      /* column slabs of the Laplacian product (1 = one pass) */
    int32_t trsv_shapes;     /* SSP_TRSV_*, as in ssp_stats */
    int32_t trsv_levels_w8, trsv_levels_w16, trsv_levels_w32;
    double ms_trsv_tune;
} ssp_solve_report;

/* ---- errors ---- */
const char* ssp_last_error(void);

/* ---- context: one device, one stream, grow-only workspace ---- */
/* The workspace is allocated and freed stream-ordered (cudaMallocAsync / cudaFreeAsync) on the context's
 * stream, so growing or releasing it never waits for the whole device. */
int ssp_context_create(int32_t device, ssp_context** ctx);
int ssp_context_destroy(ssp_context* ctx);
/* stream: a cudaStream_t (NULL = the context's own stream).  The context's frees are ordered on that stream,
 * including those of ssp_context_destroy: destroy the context before the stream it was given. */
int ssp_context_set_stream(ssp_context* ctx, void* stream);
int64_t ssp_context_kernels_launched(const ssp_context* ctx);
int64_t ssp_context_workspace_bytes(const ssp_context* ctx);
/* free the context's cached device workspace (it grows again on the next call) */
int ssp_context_release_workspace(ssp_context* ctx);

/* ---- parameters ---- */
void ssp_params_default(ssp_params* p);
void ssp_params_new(ssp_params* p, double epsilon, int32_t beta_constant, int32_t row_constant, int32_t verbose,
                    double jl_factor, double jl_scaling_factor, uint64_t sketch_seed, uint64_t sampling_seed,
                    int32_t bench, int32_t sketch_uniform, const char* output_file, int32_t streaming);
void ssp_params_cli(ssp_params* p, double epsilon, int32_t verbose, uint64_t sketch_seed, uint64_t sampling_seed,
                    int32_t bench, const char* output_file);
/* derived values (sparsifier.rs:264,272) */
int32_t ssp_params_jl_dim(const ssp_params* p, int64_t n);
double ssp_params_beta(const ssp_params* p, int64_t n);
double ssp_params_jl_scale(const ssp_params* p, int32_t k);

/* ---- drop-in for ffi::run_solve_lap (src/lib.rs:103) ----
 * shared_jl_cols: row-major num_nodes x k (FlattenedVec effective layout), k = num_cols.
 * col_ptrs/row_indices/values: the Laplacian in CSC (int32, as the bridge passes it).
 * solution_out: row-major num_nodes x k, caller-allocated.
 * Stopping rule of the reference: ||r||^2 <= 2e-7 or 400 iterations; returns
 * SSP_ERR_NOT_CONVERGED where the reference throws (relative residual >= 0.01).
 * solver_output_filename is accepted and ignored, as in the reference. */
int ssp_run_solve_lap(const double* shared_jl_cols, size_t num_rows, size_t num_cols, const int32_t* col_ptrs,
                      size_t col_ptrs_len, const int32_t* row_indices, const double* values, size_t nnz,
                      const char* solver_output_filename, int32_t num_nodes, int32_t verbose,
                      double* solution_out);

/* ---- Laplacian solve with explicit options; Y and Z row-major n x k, host or device ---- */
void ssp_solve_opts_default(ssp_solve_opts* o);
int ssp_solve_lap(ssp_context* ctx, const ssp_csc* lap, const double* Y, int32_t k, double* Z, int32_t mem,
                  const ssp_solve_opts* opts, ssp_solve_report* rep);

/* ---- sparsify one graph (input: symmetric matrix whose upper triangle holds the edges) ---- */
int ssp_sparsify(ssp_context* ctx, const ssp_csc* graph, const ssp_params* params, int32_t out_mem,
                 ssp_csc_out* out, ssp_stats* stats);
/* The same with a graph Laplacian as input (Sparsifier::from_matrix loads one, sparsifier.rs:299-300): the
 * graph is the negated off-diagonal (ssp_laplacian_to_graph), so edge (i, j) has weight -L[i][j], every edge is
 * sketched, and the result equals ssp_sparsify on that graph.  lap in host or device memory. */
int ssp_sparsify_laplacian(ssp_context* ctx, const ssp_csc* lap, const ssp_params* params, int32_t out_mem,
                           ssp_csc_out* out, ssp_stats* stats);
/* host only: the adjacency of a Laplacian, entry (i, j) = -L[i][j] for i != j, diagonal dropped, order kept
 * (host CSC out, free with ssp_csc_free) */
int ssp_laplacian_to_graph(const ssp_csc* lap, ssp_csc_out* graph);
int ssp_csc_free(ssp_csc_out* out);

/* ---- several graphs in one launch sequence (batched serving) ----
 * No counterpart in the reference, which sparsifies one graph per process and solves its right-hand sides one
 * after another (example.cc:551-568).  The count graphs (host CSCs, as for ssp_sparsify) are sparsified as
 * the disjoint union of their Laplacians: one assembly, one factorization and one all-columns PCG for the
 * batch.  Graph b keeps its own parameters where they shape its result (epsilon, beta and row constants, JL
 * rule, scale and seeds, variance correction, output_file), and every PCG scalar is kept per (graph,
 * column), so outs[b] equals ssp_sparsify of graph b alone to the solve's rounding (the kept edges match
 * unless a coin falls within that rounding of its probability).  The batch must agree on factor_seed,
 * precision, pcg_tol, pcg_abs_tol, pcg_max_iters and reweight, and use dense_threshold = 0 (the dense tail
 * looks at the whole Schur complement and would couple the graphs).  factor_max_degree is per graph: each is
 * truncated by its own test, and -1 applies the autotuner's rule to it alone (light truncation unless its
 * probe predicts more than 30 iterations), as a lone call with the same parameters does.
 * outs[b] is host memory (free with ssp_csc_free);
 * stats[b] has graph b's sizes and PCG figures, and the batch's stage times. */
int ssp_sparsify_batch(ssp_context* ctx, int32_t count, const ssp_csc* graphs, const ssp_params* params,
                       ssp_csc_out* outs, ssp_stats* stats);

/* ---- streaming: sparsify again after inserting edges (Sparsifier::insert + sparsify, sparsifier.rs:357-376,
 * 735-790) ----
 * laplacian: the current L_H (n x n, nnz may be 0); new_edges: the edges inserted since (a symmetric CSC
 * whose upper triangle holds them, as for ssp_sparsify).  As form_laplacian (sparsifier.rs:693-709) the two are
 * summed; the JL sketch covers only the new edges (the reference sketches new_entries, :736-741), the solve
 * and the sampling run over every edge of the sum.  The sum's diagonal is rebuilt from its edges (equal to
 * the reference's L_cur + L_new up to rounding). */
int ssp_sparsify_update(ssp_context* ctx, const ssp_csc* laplacian, const ssp_csc* new_edges, const ssp_params* params,
                        int32_t out_mem, ssp_csc_out* out, ssp_stats* stats);

/* ---- the JL columns split across ranks (one GPU each) ----
 * The k sketch columns are independent once the factor exists (every rank builds the same deterministic
 * factor; with factor_max_degree = -1 the choice is probed on the global columns 0..7 on every rank).
 * Phase 1, every rank: sketch the global columns [col_begin, col_end) of the k that params implies, solve
 * them, and write sq[e] = sum over those columns of (Z[v1_e, j] - Z[v2_e, j])^2 into the device buffer sq
 * (m doubles).  With sq == NULL only *m (the edge count) is computed.
 * The caller sums sq over ranks (an all-reduce), then phase 2 (on any rank) takes d_e = sqrt(sum) and runs
 * probabilities, coins, reweighting and L_H exactly as ssp_sparsify does.  d_e differs from ssp_sparsify's
 * only in the order of the final sum over columns.  Replaces the per-column loop of example.cc:551-568
 * and sparsifier.rs:565-583 when the columns live on several GPUs. */
int ssp_shard_leverage(ssp_context* ctx, const ssp_csc* graph, const ssp_params* params, int32_t col_begin,
                       int32_t col_end, double* sq, int64_t* m, ssp_stats* stats);
int ssp_shard_finish(ssp_context* ctx, const ssp_csc* graph, const ssp_params* params, const double* sq_total,
                     int32_t out_mem, ssp_csc_out* out, ssp_stats* stats);

/* ---- serving: a persistent request loop on one device ----
 * No counterpart in the reference, which sparsifies one graph per process (sparsify_dataset, lib.rs:158-168).
 * Requests of uneven size are submitted from any host thread and served by `slots` workers, each with its
 * own stream and workspace, so admitted requests overlap on the device.  A free slot admits the oldest pending
 * request whose estimated device footprint (ssp_request_footprint) fits beside those in flight within
 * hbm_budget_bytes (a younger one may go first while the oldest has waited less than 500 ms; after that the
 * oldest is admitted first); a request whose footprint alone exceeds the budget is refused at submit
 * (SSP_ERR_CAPACITY).  The slot then adds pending requests that can share its run (same epsilon, factor
 * seed, precision, PCG options and reweighting, and dense_threshold = 0), up to max_batch
 * and its share of the budget, and runs them with ssp_sparsify_batch; other requests run exactly
 * ssp_sparsify, so their result is the same as a lone call's.  Results are collected once with ssp_wait /
 * ssp_poll (which then own res->out: free it with ssp_csc_free). */
#define SSP_REQ_SPARSIFY 0
typedef struct ssp_server ssp_server;
typedef struct {
    int32_t device;
    int32_t slots;            /* requests on the device at once */
    int64_t hbm_budget_bytes; /* admission limit on in-flight footprints; <= 0: 85% of free memory at creation */
    int32_t max_pending;      /* queue length beyond which ssp_submit refuses (0: unbounded) */
    int32_t max_batch;        /* requests that may share one run (ssp_sparsify_batch); <= 1: each runs alone */
} ssp_server_opts;
typedef struct {
    int32_t kind;             /* SSP_REQ_SPARSIFY */
    ssp_csc graph;            /* host CSC; copied by ssp_submit */
    ssp_params params;        /* copied by ssp_submit (output_file too) */
    int32_t check_probes;     /* > 0: check the result inline with this many quadratic-form probes (a15) */
} ssp_request;
typedef struct {
    int32_t status;           /* the request's own status code */
    char error[256];
    ssp_csc_out out;          /* L_H on the host */
    ssp_stats stats;
    int64_t est_bytes;        /* the footprint estimate used for admission */
    double queue_ms;          /* submit -> admitted */
    double run_ms;            /* admitted -> done */
    double latency_ms;        /* submit -> done */
    int32_t slot;
    /* inline check when check_probes > 0 (ssp_probe_quadratic_form with the request's epsilon and the
     * probes seeded by its sampling_seed, and ssp_connected_components of the graph and of L_H) */
    int32_t checked;
    int64_t probe_upper_violations, probe_lower_violations;
    double probe_mean_relative_error, probe_max_relative_error;
    int64_t components_graph, components_sparsifier;
    double check_ms;
    int32_t batch;            /* requests in the run that served this one (1: it ran alone) */
} ssp_result;
typedef struct {
    int64_t submitted, completed, failed, rejected, pending;
    int32_t inflight, peak_inflight, slots;
    int32_t waiters;          /* threads inside ssp_wait / ssp_poll */
    int64_t peak_inflight_bytes, budget_bytes;
    int64_t batches;          /* runs started (a lone request or a batch) */
    int32_t peak_batch;       /* largest batch so far */
} ssp_server_info;
void ssp_server_opts_default(ssp_server_opts* opts);
int64_t ssp_request_footprint(const ssp_csc* graph, const ssp_params* params);
int ssp_server_create(const ssp_server_opts* opts, ssp_server** server);
int ssp_submit(ssp_server* server, const ssp_request* req, uint64_t* ticket);
/* timeout_ms < 0 waits without limit; SSP_ERR_PENDING if the request is not done in time */
int ssp_wait(ssp_server* server, uint64_t ticket, int64_t timeout_ms, ssp_result* res);
int ssp_poll(ssp_server* server, uint64_t ticket, ssp_result* res);
int ssp_server_info_get(ssp_server* server, ssp_server_info* info);
/* drops pending requests, lets admitted ones finish, frees uncollected results */
int ssp_server_destroy(ssp_server* server);

/* ---- checks of a Laplacian and of a sparsifier (a15) ----
 * ssp_check_laplacian      <- Sparsifier::check_diagonal        src/sparsifier.rs:806-817
 *   counts columns whose sum exceeds tol in magnitude, the largest |column sum|, and entries whose mirror
 *   (j, i) is missing or differs (exact symmetry, as sprs::is_symmetric)
 * ssp_quadratic_forms      <- Sparsifier::compute_quadratic_form src/sparsifier.rs:820-826
 *   out[j] = x_j^T L x_j for the p columns of X (column-major n x p)
 * ssp_probe_vectors        the probe vectors: X[i + n j] = 2u - 1, u uniform from Philox((i, j)) (the reference
 *                          draws uniform(-1, 1) from thread_rng, tests.rs:50-59)
 * ssp_probe_quadratic_form <- probe_quadratic_form              src/experiments.rs:88-122
 * ssp_connected_components <- petgraph connected_components in verify_ccs, src/experiments.rs:58-64
 *   over the off-diagonal nonzeros; labels (optional) = the smallest vertex of each component */
typedef struct {
    int64_t upper_bound_violations;  /* x^T L_H x >= (1 + eps) x^T L_G x */
    int64_t lower_bound_violations;  /* x^T L_H x <= (1 - eps) x^T L_G x */
    double mean_relative_error;      /* of |qH - qG| / |qG| over the probes */
    double std_dev_relative_error;   /* population standard deviation */
    double max_relative_error;
    int32_t probes;
} ssp_probe_result;
int ssp_check_laplacian(ssp_context* ctx, const ssp_csc* lap, double tol, int64_t* bad_columns,
                        double* max_abs_colsum, int64_t* asymmetric_entries);
int ssp_probe_vectors(ssp_context* ctx, int64_t n, int32_t p, uint64_t seed, int32_t mem, double* X);
int ssp_quadratic_forms(ssp_context* ctx, const ssp_csc* lap, const double* X, int32_t p, int32_t mem, double* out);
int ssp_probe_quadratic_form(ssp_context* ctx, const ssp_csc* lap_g, const ssp_csc* lap_h, double epsilon,
                             int32_t probes, uint64_t seed, ssp_probe_result* res);
int ssp_connected_components(ssp_context* ctx, const ssp_csc* m, int32_t mem, int32_t* labels, int64_t* count);

/* ---- .mtx path (sparsify_dataset) ---- */
int ssp_sparsify_mtx(const char* input_file, const char* output_file, const ssp_params* params, ssp_stats* stats);
int ssp_read_mtx(const char* path, ssp_csc_out* out);             /* host CSC, duplicates summed */
int ssp_write_mtx(const char* path, const ssp_csc* m);            /* coordinate real general */

/* ---- Matrix Market on the device (the GPU .mtx ingest / egest; replaces read_mtx / write_mtx,
 * utils.rs:149-154,189-191, whose parsing and formatting run on one host core) ----
 * ssp_read_mtx_device: the same CSC as ssp_read_mtx, parsed on the GPU (newline index, one thread per line,
 * exact decimal conversion, stable radix sort by (column, row), duplicates summed in file order).  A file
 * whose body the per-line parser cannot mirror exactly is read by the host reader instead, so both entry
 * points always return the same matrix and the same errors.  out_mem SSP_MEM_DEVICE leaves the arrays in
 * the context (owned_by_context = 1, valid until the context's next read).
 * ssp_write_mtx_device: the bytes ssp_write_mtx writes, formatted on the GPU; m in host or device memory.
 * ssp_sparsify_mtx uses both. */
int ssp_read_mtx_device(ssp_context* ctx, const char* path, int32_t out_mem, ssp_csc_out* out);
int ssp_write_mtx_device(ssp_context* ctx, const char* path, const ssp_csc* m);
/* the exact conversions those kernels use, on the host: ssp_parse_decimal returns 1 with the correctly rounded
 * binary64 of the token s[0, len) (as strtod), 0 when the token is outside the exact converter's domain
 * (more than 19 significant digits, |decimal exponent| > 38, subnormal results, inf/nan/hex), -1 on a
 * malformed token; ssp_format_g17 writes printf("%.17g", v) into buf (cap >= 33, NUL-terminated) and returns
 * its length, or -1 for values outside the device formatter's range (decimal exponent outside [-20, 38],
 * subnormals, inf, nan). */
int ssp_parse_decimal(const char* s, size_t len, double* out);
int ssp_format_g17(double v, char* buf, size_t cap);
/* ssp_format_shortest: the device formatter of the edge-list converter, on the host: v as Rust's Display writes
 * an f64 (shortest digits that read back as v, no exponent) into buf (NUL-terminated); returns the length, or -1
 * for values it leaves to the host (not finite, subnormal, outside about [1e-22, 3e38], longer than cap - 1). */
int ssp_format_shortest(double v, char* buf, size_t cap);
/* edge list ("<n> <m>" then "u v [w]" lines) -> symmetric .mtx, first weight of a repeated pair wins
 * (edge_list_to_matrix_market, src/utils.rs:413-526) */
int ssp_edgelist_to_mtx(const char* input_path, const char* output_path, double default_weight);
/* the same conversion on the GPU (edge_list_to_matrix_market, src/utils.rs:413-526): lines indexed and parsed on
 * the device, pairs sorted stably, lines formatted with Rust's f64 text; byte for byte the file
 * ssp_edgelist_to_mtx writes.  A file the device parser does not mirror (signed or 2^32+ endpoints, unusual
 * separators, malformed lines) is converted by ssp_edgelist_to_mtx instead, with its result or error;
 * *on_device (if not NULL) says which of the two wrote the file (1: the GPU). */
int ssp_edgelist_to_mtx_device(ssp_context* ctx, const char* input_path, const char* output_path,
                               double default_weight, int32_t* on_device);

/* ---- synthetic graphs (seeded, identical on every host) as symmetric host CSC ---- */
int ssp_gen_grid2d(int64_t nx, int64_t ny, double w, ssp_csc_out* out);
int ssp_gen_grid3d(int64_t nx, int64_t ny, int64_t nz, double wlog10_lo, double wlog10_hi, uint64_t seed,
                   ssp_csc_out* out);
int ssp_gen_er(int64_t n, double avg_degree, double wlo, double whi, uint64_t seed, ssp_csc_out* out);
/* R-MAT: edge_factor * 2^scale samples with quadrant probabilities (a, b, c, 1-a-b-c), self-loops dropped,
 * symmetrized and deduplicated, LogNormal(0,1) weights rounded to FP32, largest connected component only */
int ssp_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed, ssp_csc_out* out);
/* random geometric graph in the unit square, radius sqrt(avg_degree / (pi n)), weights uniform [wlo, whi] */
int ssp_gen_rgg(int64_t n, double avg_degree, double wlo, double whi, uint64_t seed, ssp_csc_out* out);

/* ---- stage entry points (device-resident, for parity tests) ---- */
/* edges of the input (v1 < v2, weights, CSC order) and L_G, copied to caller-allocated host buffers;
 * call once with v1 == NULL to obtain m and nnz(L_G). */
int ssp_stage_graph(ssp_context* ctx, const ssp_csc* graph, int64_t* m, int64_t* lap_nnz, int32_t* v1, int32_t* v2,
                    double* w, int64_t* lap_colptr, int32_t* lap_rowidx, double* lap_values);
int ssp_stage_sketch(ssp_context* ctx, int64_t n, int64_t m, const int32_t* v1, const int32_t* v2,
                     const double* w, int32_t mem, int32_t k, double scale, uint64_t seed, int32_t uniform,
                     double* Y);
/* factor of a Laplacian: column CSC of L (vertex ids, strictly lower, unit diagonal implicit), D, levels.
 * Output arrays are caller-allocated host buffers; call once with rows==NULL to get nnz. */
int ssp_stage_factor(ssp_context* ctx, const ssp_csc* lap, uint64_t seed, int64_t dense_threshold,
                     int64_t max_degree, int64_t* nnz, int64_t* colptr, int32_t* rows, double* vals, double* D,
                     int32_t* level, int32_t* num_levels);
/* M^{-1} applied to the k columns of R (host, row-major n x k) with the factor of `lap` */
int ssp_stage_precond(ssp_context* ctx, const ssp_csc* lap, uint64_t seed, int64_t dense_threshold,
                      int64_t max_degree, const double* R, int32_t k, double* Zout);
int ssp_stage_diff_norms(ssp_context* ctx, int64_t n, int64_t m, const int32_t* v1, const int32_t* v2,
                         const double* Z, int32_t k, int32_t mem, double* d);
int ssp_stage_probs(ssp_context* ctx, int64_t m, const double* w, const double* d, double beta, double denom,
                    int32_t mem, double* p);
int ssp_stage_coins(ssp_context* ctx, int64_t m, uint64_t seed, int32_t mem, double* coins);
/* the device-wide exclusive scan every stage builds its offsets with: out[i] = sum of in[0..i), out[n] = total
 * (host arrays; out has n + 1 entries) */
int ssp_stage_scan(ssp_context* ctx, const int32_t* in, int64_t n, int64_t* out);
int ssp_stage_sample_apply(ssp_context* ctx, const ssp_csc* graph, const double* p, const double* coins,
                           int32_t reweight, int32_t mem, uint8_t* keep, ssp_csc_out* out);

/* ---- allocation-free leverage stage (no counterpart in the reference) ----
 * p[e] = min(((beta*w[e]) * d_e^2) / denom, 1) with d_e = ||Z[v1[e],:] - Z[v2[e],:]||_2, the same values as
 * ssp_stage_diff_norms followed by ssp_stage_probs.  For callers that must not allocate device memory after
 * start-up -- a host whose HBM is owned by its own pool under a fixed budget, or one that cannot take the
 * device-wide synchronisation a cudaFree implies: it needs no ssp_context and calls no cudaMalloc/cudaFree.
 * All pointers are device pointers on the current device; Z is row-major n x k; the work is enqueued on
 * `stream` (a cudaStream_t, NULL = legacy default stream) and the call returns without synchronising.
 * d lives in a static device array of SSP_STATIC_SCRATCH_EDGES doubles: m above that returns
 * SSP_ERR_CAPACITY before anything is launched; nothing in it must start at zero.  The array is shared by
 * all calls on a device, so overlapping calls (two streams or threads in flight at once) race: serialise
 * them.  The first call with each device current loads the library's device code there (with CUDA's lazy
 * module loading, that is when the static array is created: a device allocation) and looks the array up
 * with cudaGetSymbolAddress, so make that first call at start-up, before any stream capture.  The address
 * is kept per device for the life of the process: after cudaDeviceReset on a device, do not call this entry
 * point on it again.  An edge with an endpoint outside [0, n) gets p = 1 (d = NaN), as ssp_stage_diff_norms
 * gives NaN for device input and rejects host input. */
#define SSP_STATIC_SCRATCH_EDGES (1 << 20)
int ssp_stage_leverage_probs_static(void* stream, int64_t n, int64_t m, const int32_t* v1, const int32_t* v2,
                                    const double* Z, int32_t k, const double* w, double beta, double denom,
                                    double* p);

#ifdef __cplusplus
}
#endif
#endif
