/*
 * ssp_oracle.c -- CPU restatement of the spec_spars sparsification path.
 *
 * TEST INFRASTRUCTURE ONLY (see ssp_oracle.h).  Compiled with
 * -ffp-contract=off so that every multiply and add rounds on its own, as the
 * reference's Rust code does and as the bit-exact CUDA kernels are written.
 */
#include "ssp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Philox4x64-10.  Constants from the published Philox description (Salmon,
 * Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11).
 * Checked in the tests against numpy.random.Philox, an independent
 * implementation of the same generator. */
void ora_philox4x64(const uint64_t ctr[4], uint64_t k0, uint64_t k1, uint64_t out[4]) {
    uint64_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += 0x9E3779B97F4A7C15ULL;
            k1 += 0xBB67AE8584CAA73BULL;
        }
        unsigned __int128 p0 = (unsigned __int128)0xD2E7470EE14C6C93ULL * c0;
        unsigned __int128 p1 = (unsigned __int128)0xCA5A826395121157ULL * c2;
        uint64_t lo0 = (uint64_t)p0, hi0 = (uint64_t)(p0 >> 64);
        uint64_t lo1 = (uint64_t)p1, hi1 = (uint64_t)(p1 >> 64);
        uint64_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline double u53(uint64_t x) { return (double)(x >> 11) * 0x1.0p-53; }

/* Sketch entry h(e,j) (without the jl scaling factor).
 * Discrete mode (reference hash_with_inputs + transform, sparsifier.rs:379-407): +-1 from one bit.
 * Uniform mode (reference hash_with_inputs_alt + u32_to_f64_minus_one_to_one, sparsifier.rs:385-420):
 * ((x + 0.5) / 2^32) * 2 - 1 of a 32-bit word.  The reference draws the bits from CityHash64; this
 * build draws them from Philox keyed by the sketch seed. */
double ora_sketch_entry(uint64_t seed, int uniform, int64_t e, int64_t j) {
    uint64_t out[4];
    if (!uniform) {
        uint64_t ctr[4] = {(uint64_t)e, (uint64_t)(j >> 8), 0, 0};
        ora_philox4x64(ctr, seed, ORA_STREAM_SIGN, out);
        uint64_t word = out[(j >> 6) & 3];
        return ((word >> (j & 63)) & 1) ? -1.0 : 1.0;
    } else {
        uint64_t ctr[4] = {(uint64_t)e, (uint64_t)(j >> 3), 0, 0};
        ora_philox4x64(ctr, seed, ORA_STREAM_UNIF, out);
        uint64_t word = out[(j >> 1) & 3];
        uint32_t x = (j & 1) ? (uint32_t)(word >> 32) : (uint32_t)word;
        const double SCALE = 4294967296.0;
        double u = ((double)x + 0.5) / SCALE;
        return 2.0 * u - 1.0;
    }
}

/* Coin for edge e (reference flip_coins, sparsifier.rs:625-633, draws from StdRng in edge order;
 * this build uses Philox keyed by the sampling seed, counter = edge index). */
double ora_coin(uint64_t seed, int64_t e) {
    uint64_t out[4];
    uint64_t ctr[4] = {(uint64_t)(e >> 2), 0, 0, 0};
    ora_philox4x64(ctr, seed, ORA_STREAM_COIN, out);
    return u53(out[e & 3]);
}

uint64_t ora_priority(uint64_t seed, int64_t v) {
    uint64_t out[4];
    uint64_t ctr[4] = {(uint64_t)v, 0, 0, 0};
    ora_philox4x64(ctr, seed, ORA_STREAM_PRIO, out);
    return out[0];
}

/* Uniform [0,1) for sample slot `slot` of column v (reference: mt19937 seeded from random_device,
 * example.cc:99-101,264). */
double ora_factor_uniform(uint64_t seed, int64_t v, int64_t slot) {
    uint64_t out[4];
    uint64_t ctr[4] = {(uint64_t)v, (uint64_t)(slot >> 2), 0, 0};
    ora_philox4x64(ctr, seed, ORA_STREAM_FACTOR, out);
    return u53(out[slot & 3]);
}

/* ------------------------------------------------------------------------ */
/* a2: edges = upper-triangle entries of the input CSC in CSC order
 * (stream.rs:44-49: `for (value,(row,col)) in iter() { if row < col { insert } }`;
 * sparsifier.rs:365 drops value == 0).  Rows must be strictly increasing per column
 * (sprs CsMat invariant).  Negative or non-finite weights are rejected (-3): the
 * reference would take sqrt of a negative number (sparsifier.rs:97). */
int64_t ora_extract_edges(int64_t n, const int64_t* colptr, const int32_t* rowidx, const double* val,
                          int32_t* v1, int32_t* v2, double* w) {
    if (n < 0 || colptr[0] != 0) return -1;
    int64_t m = 0;
    for (int64_t c = 0; c < n; c++) {
        if (colptr[c + 1] < colptr[c]) return -1;
        int32_t prev = -1;
        for (int64_t p = colptr[c]; p < colptr[c + 1]; p++) {
            int32_t r = rowidx[p];
            if (r < 0 || r >= n || r <= prev) return -2;
            prev = r;
            double x = val[p];
            if (r < c && x != 0.0) {
                if (!(x > 0.0) || !isfinite(x)) return -3;
                if (v1) { v1[m] = r; v2[m] = (int32_t)c; w[m] = x; }
                m++;
            }
        }
    }
    return m;
}

/* ------------------------------------------------------------------------ */
/* a5: L_G.  Off-diagonals -w at (v1,v2),(v2,v1); diag[v] accumulated in edge order
 * (Triplet::insert, sparsifier.rs:48-70); CSC with rows ascending (sprs to_csc);
 * diagonal entries equal to 0 (isolated vertices) are not stored (sprs add drops zeros,
 * sparsifier.rs:703). */
static void adjacency(int64_t n, int64_t m, const int32_t* v1, const int32_t* v2,
                      int64_t** ptr_out, int32_t** nbr_out, int64_t** eid_out) {
    int64_t* ptr = calloc((size_t)n + 1, sizeof(int64_t));
    for (int64_t e = 0; e < m; e++) { ptr[v1[e] + 1]++; ptr[v2[e] + 1]++; }
    for (int64_t v = 0; v < n; v++) ptr[v + 1] += ptr[v];
    int32_t* nbr = malloc(sizeof(int32_t) * (size_t)(2 * m + 1));
    int64_t* eid = malloc(sizeof(int64_t) * (size_t)(2 * m + 1));
    int64_t* cur = malloc(sizeof(int64_t) * (size_t)(n + 1));
    memcpy(cur, ptr, sizeof(int64_t) * (size_t)n);
    /* appending in edge order yields neighbour-sorted lists: a vertex's lower
     * neighbours come from its own column (ascending rows) and precede all edges of
     * later columns (its upper neighbours, ascending column). */
    for (int64_t e = 0; e < m; e++) {
        int32_t a = v1[e], b = v2[e];
        nbr[cur[a]] = b; eid[cur[a]++] = e;
        nbr[cur[b]] = a; eid[cur[b]++] = e;
    }
    free(cur);
    *ptr_out = ptr; *nbr_out = nbr; *eid_out = eid;
}

int64_t ora_laplacian_nnz(int64_t n, int64_t m, const int32_t* v1, const int32_t* v2, const double* w) {
    double* diag = calloc((size_t)n + 1, sizeof(double));
    for (int64_t e = 0; e < m; e++) { diag[v1[e]] += w[e]; diag[v2[e]] += w[e]; }
    int64_t nnz = 2 * m;
    for (int64_t v = 0; v < n; v++) nnz += (diag[v] != 0.0);
    free(diag);
    return nnz;
}

void ora_laplacian(int64_t n, int64_t m, const int32_t* v1, const int32_t* v2, const double* w,
                   int64_t* colptr, int32_t* rowidx, double* val) {
    double* diag = calloc((size_t)n + 1, sizeof(double));
    for (int64_t e = 0; e < m; e++) { diag[v1[e]] += w[e]; diag[v2[e]] += w[e]; }
    int64_t *ptr, *eid; int32_t* nbr;
    adjacency(n, m, v1, v2, &ptr, &nbr, &eid);
    int64_t q = 0;
    colptr[0] = 0;
    for (int64_t v = 0; v < n; v++) {
        int diag_done = (diag[v] == 0.0);
        for (int64_t p = ptr[v]; p < ptr[v + 1]; p++) {
            if (!diag_done && nbr[p] > v) { rowidx[q] = (int32_t)v; val[q++] = diag[v]; diag_done = 1; }
            rowidx[q] = nbr[p]; val[q++] = -w[eid[p]];
        }
        if (!diag_done) { rowidx[q] = (int32_t)v; val[q++] = diag[v]; }
        colptr[v + 1] = q;
    }
    free(ptr); free(nbr); free(eid); free(diag);
}

/* ------------------------------------------------------------------------ */
/* a4: Y = B^T Q.  Column e of B^T has -sqrt(w) at v1 and +sqrt(w) at v2
 * (sparsifier.rs:90-114).  Y[v,j] = sum over incident edges in edge order of
 * (h(e,j)*scale) * b_ev (jl_sketch_colwise, sparsifier.rs:490-506, without the
 * nondeterministic block summation of :525-527). */
void ora_sketch(int64_t n, int64_t m, const int32_t* v1, const int32_t* v2, const double* w,
                int32_t k, double scale, uint64_t seed, int uniform, double* Y) {
    int64_t *ptr, *eid; int32_t* nbr;
    adjacency(n, m, v1, v2, &ptr, &nbr, &eid);
    memset(Y, 0, sizeof(double) * (size_t)n * (size_t)k);
    for (int64_t v = 0; v < n; v++) {
        double* y = Y + v * (int64_t)k;
        for (int64_t p = ptr[v]; p < ptr[v + 1]; p++) {
            int64_t e = eid[p];
            double sw = sqrt(w[e]);
            double b = (v == v2[e]) ? sw : -sw;
            for (int32_t j = 0; j < k; j++) {
                double hs = ora_sketch_entry(seed, uniform, e, j) * scale;
                double t = hs * b;
                y[j] = y[j] + t;
            }
        }
    }
    free(ptr); free(nbr); free(eid);
}

/* ------------------------------------------------------------------------ */
/* a7: approximate Cholesky.
 *
 * Per-column arithmetic restates perform_factorization_device (example.cc:188-300):
 * gather the column's entries (original lower entries plus fill), merge equal rows
 * (:209-235), sort by value (:243), prefix sums (:248-258), then for every entry i
 * but the last draw u, pick the first j > i with c_j - c_i >= u (S - c_i) (:264-268)
 * and emit fill (max(r_i,r_j), min(r_i,r_j)) of weight v_i (S - c_i) / S (:269-271);
 * scale v_i /= S (:293), D = S (:441), L entries are -v_i/S with an implicit unit
 * diagonal (:437-446).
 *
 * Deliberate differences (all deterministic):
 *  - elimination order: increasing (priority, id) with priority = Philox(seed, v),
 *    executed level by level: a vertex is eliminated once every neighbour with a
 *    smaller key is (the reference does the same with natural order and dependency
 *    counts, example.cc:163-168,302-315, pre_process.hpp:495-512).  The factor equals
 *    sequential elimination in key order.
 *  - merge sorts by (row, weight) and sums each run left to right; the value sort
 *    breaks ties by row; prefix sums use 32-wide Kogge-Stone chunks with a
 *    sequential carry between chunks (the CUDA warp scan).
 *  - u = Philox(seed, column, slot) instead of mt19937(random_device()).
 *  - dense tail: once at most `dense_threshold` vertices are live at a level
 *    boundary and the next frontier holds at most 8 vertices (the Schur complement
 *    has become dense), the live Schur complement is merged into a dense matrix W and the
 *    remaining vertices are eliminated one per level in key order, with fill added
 *    to W in elimination order.
 */
#define ORA_DENSE_FRONTIER_MAX 8
typedef struct { int32_t u; double w; } ent_t;

typedef struct { ent_t* e; int64_t n, cap; } bag_t;

static void bag_push(bag_t* b, int32_t u, double w) {
    if (b->n == b->cap) {
        b->cap = b->cap ? 2 * b->cap : 4;
        b->e = realloc(b->e, sizeof(ent_t) * (size_t)b->cap);
    }
    b->e[b->n].u = u; b->e[b->n].w = w; b->n++;
}

static int cmp_uw(const void* a, const void* b) {
    const ent_t *x = a, *y = b;
    if (x->u != y->u) return x->u < y->u ? -1 : 1;
    if (x->w != y->w) return x->w < y->w ? -1 : 1;
    return 0;
}
static int cmp_wu(const void* a, const void* b) {
    const ent_t *x = a, *y = b;
    if (x->w != y->w) return x->w < y->w ? -1 : 1;
    if (x->u != y->u) return x->u < y->u ? -1 : 1;
    return 0;
}

/* inclusive scan: 32-wide Kogge-Stone per chunk, carry added as carry + t */
static void chunk_scan(const double* a, double* c, int64_t cnt) {
    double carry = 0.0;
    for (int64_t base = 0; base < cnt; base += 32) {
        int len = (int)((cnt - base) < 32 ? (cnt - base) : 32);
        double t[32], t2[32];
        for (int l = 0; l < 32; l++) t[l] = (l < len) ? a[base + l] : 0.0;
        for (int s = 1; s < 32; s <<= 1) {
            for (int l = 0; l < 32; l++) t2[l] = (l >= s) ? t[l - s] + t[l] : t[l];
            memcpy(t, t2, sizeof(t));
        }
        for (int l = 0; l < len; l++) c[base + l] = (base > 0) ? carry + t[l] : t[l];
        carry = c[base + len - 1];
    }
}

typedef struct {
    int32_t a, b; double w;
} fill_t;

typedef struct {
    int64_t n;
    int32_t* rows; double* vals; int64_t cnt; double D;
} col_t;

/* eliminate one column given its merged entries (sorted by (u,w) and merged already) */
static void eliminate_merged(uint64_t seed, int32_t v, ent_t* E, int64_t cnt, col_t* col,
                             fill_t** fills, int64_t* nf, int64_t* fcap) {
    col->cnt = cnt;
    if (cnt == 0) { col->D = 0.0; col->rows = NULL; col->vals = NULL; return; }
    qsort(E, (size_t)cnt, sizeof(ent_t), cmp_wu);
    double* a = calloc((size_t)cnt, sizeof(double));
    double* c = calloc((size_t)cnt, sizeof(double));
    for (int64_t i = 0; i < cnt; i++) a[i] = E[i].w;
    chunk_scan(a, c, cnt);
    double S = c[cnt - 1];
    for (int64_t i = 0; i + 1 < cnt; i++) {
        double u = ora_factor_uniform(seed, v, i);
        double rem = S - c[i];
        double tgt = u * rem;
        int64_t lo = i + 1, hi = cnt; /* lower_bound of !((c[j]-c[i]) < tgt) */
        while (lo < hi) {
            int64_t mid = lo + (hi - lo) / 2;
            if ((c[mid] - c[i]) < tgt) lo = mid + 1; else hi = mid;
        }
        int64_t j = lo < cnt ? lo : cnt - 1;
        int32_t r0 = E[i].u, r1 = E[j].u;
        double wf = (E[i].w * rem) / S;
        if (*nf == *fcap) { *fcap = *fcap ? 2 * *fcap : 64; *fills = realloc(*fills, sizeof(fill_t) * (size_t)*fcap); }
        (*fills)[*nf].a = r0 > r1 ? r0 : r1;
        (*fills)[*nf].b = r0 > r1 ? r1 : r0;
        (*fills)[*nf].w = wf;
        (*nf)++;
    }
    col->rows = malloc(sizeof(int32_t) * (size_t)cnt);
    col->vals = malloc(sizeof(double) * (size_t)cnt);
    for (int64_t i = 0; i < cnt; i++) { col->rows[i] = E[i].u; col->vals[i] = -(E[i].w / S); }
    col->D = S;
    free(a); free(c);
}

/* sort by (u,w) and merge equal u left to right; returns merged count */
static int64_t merge_entries(ent_t* E, int64_t cnt) {
    if (cnt == 0) return 0;
    qsort(E, (size_t)cnt, sizeof(ent_t), cmp_uw);
    int64_t o = 0;
    for (int64_t i = 1; i < cnt; i++) {
        if (E[i].u == E[o].u) E[o].w = E[o].w + E[i].w;
        else E[++o] = E[i];
    }
    return o + 1;
}

static uint64_t* g_prio;
static inline int key_less(int32_t a, int32_t b) {
    if (g_prio[a] != g_prio[b]) return g_prio[a] < g_prio[b];
    return a < b;
}
static int cmp_key(const void* x, const void* y) {
    int32_t a = *(const int32_t*)x, b = *(const int32_t*)y;
    if (a == b) return 0;
    return key_less(a, b) ? -1 : 1;
}
static int cmp_i32(const void* x, const void* y) {
    int32_t a = *(const int32_t*)x, b = *(const int32_t*)y;
    return (a > b) - (a < b);
}

int ora_factor(int64_t n, const int64_t* colptr, const int32_t* rowidx, const double* val,
               uint64_t seed, int64_t dense_threshold, int64_t max_degree, ora_factor_t* out) {
    memset(out, 0, sizeof(*out));
    out->n = n;
    bag_t* bag = calloc((size_t)n + 1, sizeof(bag_t));
    for (int64_t c = 0; c < n; c++)
        for (int64_t p = colptr[c]; p < colptr[c + 1]; p++) {
            int32_t r = rowidx[p];
            if (r > c) {
                double w = fabs(val[p]);
                if (w == 0.0) continue;
                bag_push(&bag[c], r, w);
                bag_push(&bag[r], (int32_t)c, w);
            }
        }
    int64_t live_entries = 0;
    for (int64_t v = 0; v < n; v++) live_entries += bag[v].n;
    uint64_t* prio = malloc(sizeof(uint64_t) * (size_t)(n + 1));
    for (int64_t v = 0; v < n; v++) prio[v] = ora_priority(seed, v);
    g_prio = prio;
    int64_t* count = calloc((size_t)n + 1, sizeof(int64_t));
    for (int64_t v = 0; v < n; v++)
        for (int64_t i = 0; i < bag[v].n; i++)
            if (key_less(bag[v].e[i].u, (int32_t)v)) count[v]++;
    char* dead = calloc((size_t)n + 1, 1);
    char* touched = calloc((size_t)n + 1, 1);
    col_t* cols = calloc((size_t)n + 1, sizeof(col_t));
    out->level = malloc(sizeof(int32_t) * (size_t)(n + 1));
    out->order = malloc(sizeof(int32_t) * (size_t)(n + 1));
    int32_t* frontier = malloc(sizeof(int32_t) * (size_t)(n + 1));
    int32_t* next = malloc(sizeof(int32_t) * (size_t)(n + 1));
    int64_t nfr = 0, nnext = 0, neliminated = 0;
    for (int64_t v = 0; v < n; v++) if (count[v] == 0) frontier[nfr++] = (int32_t)v;
    fill_t* fills = NULL; int64_t nf = 0, fcap = 0;
    int32_t lvl = 0;
    int truncated = 0;
    while (nfr > 0) {
        /* truncation: the live Schur complement is too dense to be worth eliminating */
        if (max_degree > 0 && live_entries > max_degree * (n - neliminated)) { truncated = 1; break; }
        /* dense tail once few vertices remain and the frontier has collapsed */
        if (dense_threshold > 0 && (n - neliminated) <= dense_threshold && nfr <= ORA_DENSE_FRONTIER_MAX) break;
        qsort(frontier, (size_t)nfr, sizeof(int32_t), cmp_i32);
        nf = 0;
        for (int64_t f = 0; f < nfr; f++) {
            int32_t v = frontier[f];
            /* live entries of the bag (entries to eliminated vertices are stale) */
            int64_t cnt = 0;
            ent_t* E = malloc(sizeof(ent_t) * (size_t)(bag[v].n + 1));
            for (int64_t i = 0; i < bag[v].n; i++)
                if (!dead[bag[v].e[i].u]) E[cnt++] = bag[v].e[i];
            int64_t mc = merge_entries(E, cnt);
            eliminate_merged(seed, v, E, mc, &cols[v], &fills, &nf, &fcap);
            free(E);
            live_entries -= 2 * cnt;
            out->level[v] = lvl;
            out->order[neliminated++] = v;
        }
        live_entries += 2 * nf;
        for (int64_t f = 0; f < nfr; f++) dead[frontier[f]] = 1;
        /* fill: both directions into the bags; the endpoint with the larger key counts it */
        nnext = 0;
        for (int64_t i = 0; i < nf; i++) {
            int32_t a = fills[i].a, b = fills[i].b;
            bag_push(&bag[a], b, fills[i].w);
            bag_push(&bag[b], a, fills[i].w);
            if (key_less(b, a)) count[a]++; else count[b]++;
        }
        /* release: every live entry of an eliminated bag decrements its endpoint */
        for (int64_t f = 0; f < nfr; f++) {
            int32_t v = frontier[f];
            for (int64_t i = 0; i < bag[v].n; i++) {
                int32_t u = bag[v].e[i].u;
                if (dead[u]) continue;
                count[u]--;
                if (!touched[u]) { touched[u] = 1; next[nnext++] = u; }
            }
        }
        int64_t k2 = 0;
        for (int64_t i = 0; i < nnext; i++) {
            int32_t u = next[i];
            touched[u] = 0;
            if (count[u] == 0) frontier[k2++] = u;
        }
        nfr = k2;
        lvl++;
    }
    out->dense_start = (int32_t)neliminated;
    if (truncated) {
        /* remaining vertices: one final level, no L entries, D = sum of the merged live weights (row order) */
        int32_t* rem = malloc(sizeof(int32_t) * (size_t)(n - neliminated + 1));
        int64_t t = 0;
        for (int64_t v = 0; v < n; v++) if (!dead[v]) rem[t++] = (int32_t)v;
        for (int64_t i = 0; i < t; i++) {
            int32_t v = rem[i];
            int64_t cnt = 0;
            ent_t* E = malloc(sizeof(ent_t) * (size_t)(bag[v].n + 1));
            for (int64_t q = 0; q < bag[v].n; q++)
                if (!dead[bag[v].e[q].u]) E[cnt++] = bag[v].e[q];
            int64_t mc = merge_entries(E, cnt);
            double d = 0.0;
            for (int64_t q = 0; q < mc; q++) d = d + E[q].w;
            free(E);
            cols[v].cnt = 0; cols[v].rows = NULL; cols[v].vals = NULL; cols[v].D = d;
            out->level[v] = lvl;
            out->order[neliminated++] = v;
        }
        free(rem);
        lvl++;
    } else if (neliminated < n) {
        /* dense tail */
        int64_t T = n - neliminated;
        int32_t* rem = malloc(sizeof(int32_t) * (size_t)T);
        int64_t t = 0;
        for (int64_t v = 0; v < n; v++) if (!dead[v]) rem[t++] = (int32_t)v;
        qsort(rem, (size_t)T, sizeof(int32_t), cmp_key);
        int64_t* idx = malloc(sizeof(int64_t) * (size_t)n);
        for (int64_t i = 0; i < T; i++) idx[rem[i]] = i;
        double* W = calloc((size_t)(T * T), sizeof(double));
        for (int64_t i = 0; i < T; i++) {
            int32_t v = rem[i];
            int64_t cnt = 0;
            ent_t* E = malloc(sizeof(ent_t) * (size_t)(bag[v].n + 1));
            for (int64_t q = 0; q < bag[v].n; q++)
                if (!dead[bag[v].e[q].u]) E[cnt++] = bag[v].e[q];
            int64_t mc = merge_entries(E, cnt);
            for (int64_t q = 0; q < mc; q++) W[i * T + idx[E[q].u]] = E[q].w;
            free(E);
        }
        ent_t* E = malloc(sizeof(ent_t) * (size_t)(T + 1));
        for (int64_t i = 0; i < T; i++) {
            int32_t v = rem[i];
            int64_t cnt = 0;
            for (int64_t q = i + 1; q < T; q++) {
                double x = W[i * T + q];
                if (x != 0.0) { E[cnt].u = rem[q]; E[cnt].w = x; cnt++; }
            }
            nf = 0;
            eliminate_merged(seed, v, E, cnt, &cols[v], &fills, &nf, &fcap);
            for (int64_t q = 0; q < nf; q++) {
                int64_t ia = idx[fills[q].a], ib = idx[fills[q].b];
                W[ia * T + ib] = W[ia * T + ib] + fills[q].w;
                W[ib * T + ia] = W[ib * T + ia] + fills[q].w;
            }
            out->level[v] = lvl++;
            out->order[neliminated++] = v;
        }
        free(E); free(W); free(idx); free(rem);
    }
    out->num_levels = lvl;
    /* pack CSC */
    out->colstart = malloc(sizeof(int64_t) * (size_t)(n + 1));
    out->colstart[0] = 0;
    for (int64_t v = 0; v < n; v++) out->colstart[v + 1] = out->colstart[v] + cols[v].cnt;
    out->nnz = out->colstart[n];
    out->rows = malloc(sizeof(int32_t) * (size_t)(out->nnz + 1));
    out->vals = malloc(sizeof(double) * (size_t)(out->nnz + 1));
    out->D = malloc(sizeof(double) * (size_t)(n + 1));
    for (int64_t v = 0; v < n; v++) {
        if (cols[v].cnt) {
            memcpy(out->rows + out->colstart[v], cols[v].rows, sizeof(int32_t) * (size_t)cols[v].cnt);
            memcpy(out->vals + out->colstart[v], cols[v].vals, sizeof(double) * (size_t)cols[v].cnt);
        }
        out->D[v] = cols[v].D;
        free(cols[v].rows); free(cols[v].vals);
    }
    for (int64_t v = 0; v < n; v++) free(bag[v].e);
    free(bag); free(prio); free(count); free(dead); free(touched); free(cols);
    free(frontier); free(next); free(fills);
    g_prio = NULL;
    return 0;
}

void ora_factor_free(ora_factor_t* f) {
    free(f->colstart); free(f->rows); free(f->vals); free(f->D); free(f->level); free(f->order);
    memset(f, 0, sizeof(*f));
}

int64_t ora_factor_nnz(const ora_factor_t* f) { return f->nnz; }

void ora_factor_export(const ora_factor_t* f, int64_t* colstart, int32_t* rows, double* vals, double* D,
                       int32_t* level, int32_t* order) {
    memcpy(colstart, f->colstart, sizeof(int64_t) * (size_t)(f->n + 1));
    memcpy(rows, f->rows, sizeof(int32_t) * (size_t)f->nnz);
    memcpy(vals, f->vals, sizeof(double) * (size_t)f->nnz);
    memcpy(D, f->D, sizeof(double) * (size_t)f->n);
    memcpy(level, f->level, sizeof(int32_t) * (size_t)f->n);
    memcpy(order, f->order, sizeof(int32_t) * (size_t)f->n);
}

/* ------------------------------------------------------------------------ */
/* M^{-1} r: forward solve with L (columns in elimination order), scale by D
 * skipping zero pivots, backward solve with L^T (custom_cg.hpp:224-235). */
void ora_precond(const ora_factor_t* f, const double* r, double* z) {
    int64_t n = f->n;
    double* y = malloc(sizeof(double) * (size_t)(n + 1));
    memcpy(y, r, sizeof(double) * (size_t)n);
    for (int64_t t = 0; t < n; t++) {
        int32_t v = f->order[t];
        double yv = y[v];
        for (int64_t p = f->colstart[v]; p < f->colstart[v + 1]; p++) y[f->rows[p]] -= f->vals[p] * yv;
    }
    for (int64_t v = 0; v < n; v++) z[v] = (f->D[v] != 0.0) ? y[v] / f->D[v] : y[v];
    for (int64_t t = n - 1; t >= 0; t--) {
        int32_t v = f->order[t];
        double s = z[v];
        for (int64_t p = f->colstart[v]; p < f->colstart[v + 1]; p++) s -= f->vals[p] * z[f->rows[p]];
        z[v] = s;
    }
    free(y);
}

static void spmv(int64_t n, const int64_t* cp, const int32_t* ri, const double* va, const double* x, double* y) {
    for (int64_t c = 0; c < n; c++) {
        double s = 0.0;
        for (int64_t p = cp[c]; p < cp[c + 1]; p++) s += va[p] * x[ri[p]];
        y[c] = s;
    }
}
static double dot(int64_t n, const double* a, const double* b) {
    double s = 0.0;
    for (int64_t i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

/* a8: PCG for each RHS column (custom_cg.hpp:96-274): b = rhs - mean(rhs) (:132), x0 = 0 (:140),
 * preconditioned CG; the reference stops on ||r||^2 <= 2e-7 (:159,213) and reports success iff
 * ||b - A x|| / ||b|| < 0.01 (:251-258).  Here the stop is ||r|| <= max(abs_tol, tol ||b||). */
int ora_pcg(int64_t n, const int64_t* cp, const int32_t* ri, const double* va, const ora_factor_t* f,
            const double* Y, int32_t k, double tol, double abs_tol, int32_t max_iters, double* Z,
            int32_t* iters, double* relres) {
    double *b = malloc(8 * (size_t)n), *x = malloc(8 * (size_t)n), *r = malloc(8 * (size_t)n),
           *z = malloc(8 * (size_t)n), *p = malloc(8 * (size_t)n), *q = malloc(8 * (size_t)n);
    int rc = 0;
    for (int32_t j = 0; j < k; j++) {
        double s = 0.0;
        for (int64_t i = 0; i < n; i++) s += Y[i * k + j];
        double mean = s / (double)n;
        for (int64_t i = 0; i < n; i++) { b[i] = Y[i * k + j] - mean; x[i] = 0.0; r[i] = b[i]; }
        double bnorm = sqrt(dot(n, b, b));
        double thr = tol * bnorm; if (abs_tol > thr) thr = abs_tol;
        int32_t it = 0;
        if (sqrt(dot(n, r, r)) > thr) {
            ora_precond(f, r, z);
            memcpy(p, z, 8 * (size_t)n);
            double rz = dot(n, r, z);
            while (it < max_iters) {
                spmv(n, cp, ri, va, p, q);
                double alpha = rz / dot(n, p, q);
                for (int64_t i = 0; i < n; i++) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; }
                it++;
                if (sqrt(dot(n, r, r)) <= thr) break;
                ora_precond(f, r, z);
                double rz2 = dot(n, r, z);
                double beta = rz2 / rz;
                rz = rz2;
                for (int64_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
            }
        }
        spmv(n, cp, ri, va, x, q);
        double rr = 0.0;
        for (int64_t i = 0; i < n; i++) { double d = b[i] - q[i]; rr += d * d; }
        double rel = bnorm > 0.0 ? sqrt(rr) / bnorm : 0.0;
        if (iters) iters[j] = it;
        if (relres) relres[j] = rel;
        if (!(rel < 0.01)) rc = 1;
        for (int64_t i = 0; i < n; i++) Z[i * k + j] = x[i];
    }
    free(b); free(x); free(r); free(z); free(p); free(q);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* a9: d_e = ||Z[v1] - Z[v2]|| (sparsifier.rs:565-583).  Reduction order fixed to the CUDA
 * kernels' (the 32-column tiles of the device layout): for each tile T, lane l squares the
 * difference in column 32T + l (0 past k), the 32 squares are summed by an xor butterfly
 * (16,8,4,2,1; lane 0's result), and the tile sums are added in tile order from 0. */
void ora_diff_norms(int64_t n, int64_t m, const int32_t* v1, const int32_t* v2, const double* Z,
                    int32_t k, int64_t ldz, double* d) {
    (void)n;
    for (int64_t e = 0; e < m; e++) {
        const double* za = Z + (int64_t)v1[e] * ldz;
        const double* zb = Z + (int64_t)v2[e] * ldz;
        double acc = 0.0;
        for (int32_t j0 = 0; j0 < k; j0 += 32) {
            double s[32], t[32];
            for (int l = 0; l < 32; l++) {
                const double x = j0 + l < k ? za[j0 + l] - zb[j0 + l] : 0.0;
                s[l] = x * x;
            }
            for (int h = 16; h >= 1; h >>= 1) {
                for (int l = 0; l < 32; l++) t[l] = s[l] + s[l ^ h];
                memcpy(s, t, sizeof(s));
            }
            acc = acc + s[0];
        }
        d[e] = sqrt(acc);
    }
}

/* a10: p_e = min(beta * w * d^2 / denom, 1) (sparsifier.rs:553: beta * -1 * value * d.powi(2) / k). */
void ora_probs(int64_t m, const double* w, const double* d, double beta, double denom, double* p) {
    for (int64_t e = 0; e < m; e++) {
        double d2 = d[e] * d[e];
        double x = ((beta * w[e]) * d2) / denom;
        p[e] = (x < 1.0) ? x : 1.0;
        if (x != x) p[e] = 1.0;
    }
}

/* a11/a12: keep iff coin < p (:639); kept weight w/sqrt(p) (:657) or w/p; the
 * reweighting triplets (:661,:667) are added to L_G (:682-691) and exact zeros drop. */
int64_t ora_sample_apply(int64_t n, int64_t m, const int32_t* v1, const int32_t* v2, const double* w,
                         const double* p, const double* coins, int reweight,
                         const int64_t* lg_cp, const int32_t* lg_ri, const double* lg_va,
                         int64_t* lh_cp, int32_t* lh_ri, double* lh_va, uint8_t* keep) {
    double* dchange = calloc((size_t)n + 1, sizeof(double));
    double* offchange = malloc(sizeof(double) * (size_t)(m + 1));
    for (int64_t e = 0; e < m; e++) {
        int kept = coins[e] < p[e];
        if (keep) keep[e] = (uint8_t)kept;
        double X;
        if (kept) {
            double t = reweight ? w[e] / p[e] : w[e] / sqrt(p[e]);
            double change = w[e] - t;
            X = change * -1.0;
        } else {
            X = w[e] * -1.0;
        }
        offchange[e] = X * -1.0;
        dchange[v1[e]] += X;
        dchange[v2[e]] += X;
    }
    /* edge id lookup for off-diagonal (a,b): edges are unique per pair; build adjacency */
    int64_t *ptr, *eid; int32_t* nbr;
    adjacency(n, m, v1, v2, &ptr, &nbr, &eid);
    int64_t q = 0;
    if (lh_cp) lh_cp[0] = 0;
    for (int64_t c = 0; c < n; c++) {
        int64_t a = ptr[c];
        for (int64_t t = lg_cp[c]; t < lg_cp[c + 1]; t++) {
            int32_t r = lg_ri[t];
            double x;
            if (r == c) {
                x = lg_va[t] + dchange[c];
            } else {
                while (a < ptr[c + 1] && nbr[a] < r) a++;
                x = lg_va[t] + offchange[eid[a]];
            }
            if (x != 0.0) {
                if (lh_ri) { lh_ri[q] = r; lh_va[q] = x; }
                q++;
            }
        }
        if (lh_cp) lh_cp[c + 1] = q;
    }
    free(ptr); free(nbr); free(eid); free(dchange); free(offchange);
    return q;
}

/* ------------------------------------------------------------------------ */
/* Synthetic ER workload (the same graph as the library's generator; see the header). */
#define ORA_STREAM_GEN 0x47454e31ULL
static double gen_u53(uint64_t seed, uint64_t a, uint64_t b) {
    uint64_t ctr[4] = {a, b, 0, 0}, out[4];
    ora_philox4x64(ctr, seed, ORA_STREAM_GEN, out);
    return u53(out[0]);
}

int64_t ora_gen_er(int64_t n, double avg_degree, double wlo, double whi, uint64_t seed, int32_t* v1, int32_t* v2,
                   double* w, int64_t cap) {
    if (n < 2) return 0;
    double p = avg_degree / (double)(n - 1);
    if (p > 1.0) p = 1.0;
    const double lp = log1p(-p);
    int64_t v = 1, u = -1, m = 0;
    uint64_t draw = 0;
    while (v < n) {
        const double x = gen_u53(seed, draw++, 0);
        const int64_t skip = (p >= 1.0) ? 0 : (int64_t)floor(log1p(-x) / lp);
        u += 1 + skip;
        while (u >= v && v < n) {
            u -= v;
            v++;
        }
        if (v < n) {
            const double uw = gen_u53(seed, draw++, 1);
            if (v1) {
                if (m >= cap) return -1;
                v1[m] = (int32_t)u;
                v2[m] = (int32_t)v;
                w[m] = (double)(float)(wlo + (whi - wlo) * uw);
            }
            m++;
        }
    }
    return m;
}
