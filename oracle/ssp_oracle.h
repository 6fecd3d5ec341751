/*
 * ssp_oracle.h -- CPU restatement of the spec_spars sparsification path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links this code;
 * only the test-suite, __graft_entry__.smoke() and bench.py's cpu_baseline leg
 * load it (through ctypes), as the checker.  Everything is FP64 and single
 * threaded, with fixed summation orders, so that the CUDA path can be compared
 * bit-for-bit where the algorithm is integer/deterministic and within a stated
 * tolerance where it is an iterative FP solve.
 *
 * Each function cites the reference (tenchd/spec_spars) file:line it restates.
 * Where this build deliberately differs from the reference (counter-based
 * Philox randomness, a seeded random elimination order, fixed reduction
 * orders), the comment says so.
 */
#ifndef SSP_ORACLE_H
#define SSP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- counter-based RNG: Philox4x64-10 (Salmon et al., SC'11) ---- */
void ora_philox4x64(const uint64_t ctr[4], uint64_t key0, uint64_t key1, uint64_t out[4]);

/* stream identifiers (second key word) */
#define ORA_STREAM_SIGN   0x5349474eULL
#define ORA_STREAM_UNIF   0x554e4946ULL
#define ORA_STREAM_FACTOR 0x46414354ULL
#define ORA_STREAM_PRIO   0x5052494fULL
#define ORA_STREAM_COIN   0x434f494eULL

double ora_sketch_entry(uint64_t seed, int uniform, int64_t e, int64_t j);
double ora_coin(uint64_t seed, int64_t e);
uint64_t ora_priority(uint64_t seed, int64_t v);
double ora_factor_uniform(uint64_t seed, int64_t v, int64_t slot);

/* ---- a2: edge extraction, stream.rs:44-49 + sparsifier.rs:357-376 ---- */
/* Returns m (>=0) or a negative error.  Edges are upper-triangle entries
 * (row < col) with value != 0, in CSC iteration order. */
int64_t ora_extract_edges(int64_t n, const int64_t* colptr, const int32_t* rowidx,
                          const double* val, int32_t* v1, int32_t* v2, double* w);

/* ---- a5: Laplacian, sparsifier.rs:48-87,693-709 ---- */
/* nnz of L_G given edges (no explicit zeros kept) */
int64_t ora_laplacian_nnz(int64_t n, int64_t m, const int32_t* v1, const int32_t* v2, const double* w);
void ora_laplacian(int64_t n, int64_t m, const int32_t* v1, const int32_t* v2, const double* w,
                   int64_t* colptr, int32_t* rowidx, double* val);

/* ---- a4: JL sketch Y = B^T Q, sparsifier.rs:379-539 (Philox signs) ---- */
void ora_sketch(int64_t n, int64_t m, const int32_t* v1, const int32_t* v2, const double* w,
                int32_t k, double scale, uint64_t seed, int uniform, double* Y /* n x k row-major */);

/* ---- a7: approximate Cholesky, example.cc:91-323,422-469 ---- */
typedef struct {
    int64_t n;
    int64_t nnz;          /* stored off-diagonal entries of L (all columns) */
    int64_t* colstart;    /* [n+1] CSC of L (strictly lower part, unit diagonal implicit), columns = vertex ids */
    int32_t* rows;        /* [nnz] row vertex ids */
    double* vals;         /* [nnz] L entries (negative) */
    double* D;            /* [n] pivots */
    int32_t* level;       /* [n] dependency level of each vertex */
    int32_t* order;       /* [n] elimination order (vertex ids) */
    int32_t num_levels;
    int32_t dense_start;  /* number of vertices eliminated in the sparse phase */
} ora_factor_t;

/* Lower-triangle input: CSC of L_G (full), only entries with row > col are used, |value| is the weight
 * (pre_process.hpp:734-812).  dense_threshold: switch to the dense sequential phase once at most this
 * many vertices are live at a level boundary and the frontier holds at most 8 vertices (0 = never). */
/* max_degree: at a level boundary, once the live entries exceed max_degree times the live vertices
 * (average Schur-complement degree), stop: every remaining vertex goes into one final level with no L
 * entries and D = the sum of its merged live weights in row order (0 = eliminate everything). */
int ora_factor(int64_t n, const int64_t* colptr, const int32_t* rowidx, const double* val,
               uint64_t seed, int64_t dense_threshold, int64_t max_degree, ora_factor_t* out);
void ora_factor_free(ora_factor_t* f);
/* accessors for ctypes */
int64_t ora_factor_nnz(const ora_factor_t* f);
void ora_factor_export(const ora_factor_t* f, int64_t* colstart, int32_t* rows, double* vals, double* D,
                       int32_t* level, int32_t* order);

/* ---- preconditioner application M^{-1} r = L^{-T} D^+ L^{-1} r, custom_cg.hpp:224-235 ---- */
void ora_precond(const ora_factor_t* f, const double* r, double* z);

/* ---- a8: PCG per RHS, custom_cg.hpp:96-274 ---- */
/* A: full Laplacian CSC (== CSR).  Y, Z row-major n x k.  Stops a column when
 * ||r|| <= max(abs_tol, tol*||b||) or after max_iters.  iters/relres per column. */
int ora_pcg(int64_t n, const int64_t* colptr, const int32_t* rowidx, const double* val,
            const ora_factor_t* f, const double* Y, int32_t k, double tol, double abs_tol, int32_t max_iters,
            double* Z, int32_t* iters, double* relres);

/* ---- a9: diff norms, sparsifier.rs:565-583 (fixed 32-lane reduction order) ---- */
void ora_diff_norms(int64_t n, int64_t m, const int32_t* v1, const int32_t* v2, const double* Z,
                    int32_t k, int64_t ldz, double* d);

/* ---- a10: probabilities, sparsifier.rs:542-562 ---- */
void ora_probs(int64_t m, const double* w, const double* d, double beta, double denom, double* p);

/* ---- a11/a12: coins, sample, reweight, apply, sparsifier.rs:625-691 ---- */
/* reweight: 0 = w/sqrt(p) (reference), 1 = w/p.  Returns nnz of L_H; if out arrays are NULL only counts. */
int64_t ora_sample_apply(int64_t n, int64_t m, const int32_t* v1, const int32_t* v2, const double* w,
                         const double* p, const double* coins, int reweight,
                         const int64_t* lg_colptr, const int32_t* lg_rowidx, const double* lg_val,
                         int64_t* lh_colptr, int32_t* lh_rowidx, double* lh_val, uint8_t* keep);

/* Synthetic Erdos-Renyi G(n, p = avg_degree / (n - 1)) edge list, generated exactly as the library's
 * ssp_gen_er (Batagelj-Brandes geometric skipping over pairs (w < v) in order of v then w, uniforms from
 * Philox(seed, draw, 0|1) of the generator stream, weights U[wlo, whi] rounded to FP32), so that the CPU
 * baselines build their samples without loading the library.  Edges come in CSC-upper order (v1 < v2,
 * ascending v2, then v1), the order edge extraction produces.  With v1 == NULL only the count is returned;
 * otherwise at most cap edges are written and -1 is returned when more exist. */
int64_t ora_gen_er(int64_t n, double avg_degree, double wlo, double whi, uint64_t seed, int32_t* v1, int32_t* v2,
                   double* w, int64_t cap);

#ifdef __cplusplus
}
#endif
#endif
