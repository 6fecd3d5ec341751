// ssp_api.cu -- extern "C" entry points (include/specspars.h).
//
// Sparsifier flow (Sparsifier::sparsify, sparsifier.rs:722-770): edges and L_G from the input
// matrix (a2/a3/a5) -> JL sketch (a4) -> approximate Cholesky (a7) -> PCG on all k columns (a8,
// the ffi::run_solve_lap call of get_probs, sparsifier.rs:593) -> diff norms (a9) -> probabilities
// (a10) -> coins, reweighting and L_H (a11/a12).  Every stage runs on the device; there is no CPU
// fallback.  C++ exceptions never cross this boundary: each entry point returns a status code and
// records a message for ssp_last_error().
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "ssp_decimal.cuh"
#include "ssp_host.h"
#include "ssp_internal.cuh"

struct ssp_context {
    ssp::Context ctx;
};

namespace ssp {

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }

template <class Fn>
static int guarded(Fn&& fn) {
    try {
        fn();
        return SSP_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return SSP_ERR_NOMEM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return SSP_ERR_INVALID;
    }
}

static void init_context(Context& C, int device) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        throw Error(SSP_ERR_NO_DEVICE, "no CUDA device visible");
    }
    SSP_REQUIRE(device >= 0 && device < count, SSP_ERR_INVALID, "device index out of range");
    C.device = device;
    SSP_CUDA(cudaSetDevice(device));
    SSP_CUDA(cudaStreamCreateWithFlags(&C.stream, cudaStreamNonBlocking));
    C.own_stream = true;
    C.ws.set_stream(C.stream);
    SSP_CUDA(cudaMallocHost(&C.h_pinned, 64 * sizeof(int64_t)));
}

static void destroy_context(Context& C) {
    cudaSetDevice(C.device);
    if (C.stream) cudaStreamSynchronize(C.stream);
    C.ws.release();  // stream-ordered frees: wait for them before the stream goes
    if (C.stream) cudaStreamSynchronize(C.stream);
    C.ws.set_stream(nullptr);
    release_staging(C);
    if (C.h_pinned) cudaFreeHost(C.h_pinned);
    if (C.own_stream && C.stream) cudaStreamDestroy(C.stream);
    C.h_pinned = nullptr;
    C.stream = nullptr;
}

// process-wide default context for the reference-shaped entry points that carry none
static std::mutex g_default_mu;
static ssp_context* g_default = nullptr;
static Context& default_context() {
    if (!g_default) {
        auto* c = new ssp_context();
        try {
            init_context(c->ctx, 0);
        } catch (...) {
            delete c;
            throw;
        }
        g_default = c;
    }
    cudaSetDevice(g_default->ctx.device);
    return g_default->ctx;
}

// device copy of a CSC (or pass-through when already on the device)
struct DevCsc {
    int64_t n = 0, nnz = 0;
    const int64_t* colptr = nullptr;
    const int32_t* rowidx = nullptr;
    const double* val = nullptr;
};
static DevCsc to_device(Context& C, const ssp_csc* m, const char* tag) {
    SSP_REQUIRE(m && m->n > 0 && m->nnz >= 0 && m->colptr && (m->nnz == 0 || (m->rowidx && m->values)),
                SSP_ERR_INVALID, "invalid CSC descriptor");
    SSP_REQUIRE(m->n < (int64_t)INT32_MAX, SSP_ERR_INVALID, "n must be < 2^31");
    DevCsc d;
    d.n = m->n;
    d.nnz = m->nnz;
    if (m->mem == SSP_MEM_DEVICE) {
        d.colptr = m->colptr;
        d.rowidx = m->rowidx;
        d.val = m->values;
        return d;
    }
    SSP_REQUIRE(m->colptr[0] == 0 && m->colptr[m->n] == m->nnz, SSP_ERR_INVALID,
                "CSC colptr must start at 0 and end at nnz");
    std::string t(tag);
    int64_t* cp = C.ws.get_t<int64_t>(t + "_cp", m->n + 1);
    int32_t* ri = C.ws.get_t<int32_t>(t + "_ri", m->nnz + 1);
    double* va = C.ws.get_t<double>(t + "_va", m->nnz + 1);
    copy_h2d(C, cp, m->colptr, sizeof(int64_t) * (m->n + 1));
    if (m->nnz) {
        copy_h2d(C, ri, m->rowidx, sizeof(int32_t) * m->nnz);
        copy_h2d(C, va, m->values, sizeof(double) * m->nnz);
    }
    d.colptr = cp;
    d.rowidx = ri;
    d.val = va;
    return d;
}

// ---------------------------------------------------------------- parameters
static int32_t jl_dim(const ssp_params* p, int64_t n) {
    if (p->jl_dim_override > 0) return p->jl_dim_override;
    double k;
    if (p->jl_dim_rule == SSP_JL_DIM_24) k = std::ceil(24.0 * std::log((double)n) / (p->epsilon * p->epsilon));
    else k = std::ceil(std::log2((double)n) * p->jl_factor);
    if (k < 1) k = 1;
    return (int32_t)k;
}
static double jl_scale(const ssp_params* p, int32_t k) {
    return p->jl_scale_rule == SSP_JL_SCALE_INV_SQRT_K ? 1.0 / std::sqrt((double)k) : p->jl_scaling_factor;
}
static double beta_of(const ssp_params* p, int64_t n) {
    return std::pow(p->epsilon, -2.0) * (double)p->beta_constant * std::log((double)n);
}

// events for per-stage timing
struct StageTimer {
    Context& C;
    std::vector<cudaEvent_t> ev;
    explicit StageTimer(Context& c) : C(c) {}
    void mark() {
        cudaEvent_t e;
        SSP_CUDA(cudaEventCreate(&e));
        SSP_CUDA(cudaEventRecord(e, C.stream));
        ev.push_back(e);
    }
    double ms(size_t a, size_t b) {
        float t = 0;
        cudaEventElapsedTime(&t, ev[a], ev[b]);
        return t;
    }
    ~StageTimer() {
        for (auto e : ev) cudaEventDestroy(e);
    }
};

__global__ void k_count_diag(int64_t n, const int64_t* ptr, const int32_t* idx, int64_t* out) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        for (int64_t p = ptr[v]; p < ptr[v + 1]; p++)
            if (idx[p] == v) atomicAdd((unsigned long long*)out, 1ull);
}

// Splitting the JL columns across ranks (multi-GPU): phase 1 solves the global columns
// [col_lo, col_hi) and leaves the per-edge sums of squared differences in sq_out; the caller sums them
// over ranks; phase 2 takes the summed squares (sq_in) and runs probabilities, coins and L_H.
// A streaming update (ssp_sparsify_update) instead sketches only the edges inserted since the last
// sparsification (sketch_graph) while solving and sampling over the whole current graph.
struct ShardArgs {
    int32_t col_lo = 0, col_hi = 0;
    double* sq_out = nullptr;
    const double* sq_in = nullptr;
    const DevGraph* sketch_graph = nullptr;
};

// Host output of a large sparsify: the L_H arrays are allocated and their pages touched on a host thread while
// the device works (L_H has at most nnz(L_G) entries: it only reweights or drops edges of G), so the final
// device-to-host copy lands in resident pages (4.8 GB/s into fresh pages against 11 GB/s at ER n = 1M).
struct HostOutBuffers {
    std::thread th;
    int64_t* colptr = nullptr;
    int32_t* rowidx = nullptr;
    double* values = nullptr;
    int64_t cap = 0;
    void start(int64_t n, int64_t nnz_cap) {
        cap = nnz_cap;
        th = std::thread([this, n] {
            colptr = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
            rowidx = (int32_t*)malloc(sizeof(int32_t) * (cap + 1));
            values = (double*)malloc(sizeof(double) * (cap + 1));
            if (colptr) memset(colptr, 0, sizeof(int64_t) * (n + 1));
            if (rowidx) memset(rowidx, 0, sizeof(int32_t) * (cap + 1));
            if (values) memset(values, 0, sizeof(double) * (cap + 1));
        });
    }
    void join() {
        if (th.joinable()) th.join();
    }
    ~HostOutBuffers() {
        join();
        free(colptr);
        free(rowidx);
        free(values);
    }
};
constexpr int64_t HOST_OUT_PREFAULT_MIN = 1 << 20;  // entries; smaller outputs allocate at the end

// Columns solved per pass.  The PCG holds six n x ld FP64 blocks (sketch, x, r, z, p, q; the mixed mode adds
// five FP32 blocks and an FP64 increment), which for the R-MAT configuration (scale 22, eps 0.3: k = 3917)
// need 450 GB.  The columns are independent once the factor exists, so they are solved in batches of whole
// 32-column tiles.  Whether to batch is decided before the factorization with room set aside for it (70 % of
// the free memory, less 40 B per Laplacian entry and 48 B per edge); the batch size after it, from the memory
// then free (80 %, less the per-edge arrays).  SSP_COLUMN_BATCH=<columns> sets the batch.
static double column_bytes(int64_t n, int32_t precision) {
    return (double)n * (8.0 * 6 + (precision == SSP_PRECISION_MIXED ? 4.0 * 5 + 8.0 : 0.0));
}
static int32_t forced_batch(int32_t k) {
    if (const char* e = getenv("SSP_COLUMN_BATCH")) {
        const int b = atoi(e);
        if (b > 0) return std::min<int32_t>(k, std::max<int32_t>(SSP_TILE, b / SSP_TILE * SSP_TILE));
    }
    return 0;
}
static double free_for_solve(Context& C) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        cudaGetLastError();
        return 1e300;
    }
    // memory the device's default pool holds but does not use (stream-ordered frees) is free to this context
    cudaMemPool_t pool;
    uint64_t reserved = 0, used = 0;
    if (cudaDeviceGetDefaultMemPool(&pool, C.device) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
        fr += (size_t)(reserved - used);
    cudaGetLastError();
    // the solve's own buffers from an earlier call are reused
    return (double)fr + (double)(C.ws.bytes_with_prefix("sp_Y") + C.ws.bytes_with_prefix("pcg"));
}
static bool columns_fit(Context& C, const DevGraph& G, int32_t k, int32_t precision) {
    const double need = column_bytes(G.n, precision) * (double)tile_ld(k);
    return need <= 0.7 * free_for_solve(C) - 40.0 * (double)G.lap_nnz - 48.0 * (double)G.m;
}
static int32_t batch_after_factor(Context& C, const DevGraph& G, int32_t k, int32_t precision) {
    const double avail = 0.8 * free_for_solve(C) - 48.0 * (double)G.m - (1.0 * (1 << 30));
    const int64_t cols = (int64_t)(avail / column_bytes(G.n, precision)) / SSP_TILE * SSP_TILE;
    return (int32_t)std::max<int64_t>(SSP_TILE, std::min<int64_t>(cols, k));
}

// the preconditioner's level-launch shapes (ssp_stats / ssp_solve_report share the field names)
template <class S>
static void copy_trsv_stats(S& s, const PcgReport& r) {
    s.trsv_shapes = r.trsv_shapes;
    s.trsv_levels_w8 = r.trsv_levels[0];
    s.trsv_levels_w16 = r.trsv_levels[1];
    s.trsv_levels_w32 = r.trsv_levels[2];
    s.ms_trsv_tune = r.ms_trsv_tune;
}

static void merge_report(PcgReport& a, const PcgReport& b, int32_t ka, int32_t kb) {
    a.mean_iters = (a.mean_iters * ka + b.mean_iters * kb) / (double)(ka + kb);
    a.max_iters_used = std::max(a.max_iters_used, b.max_iters_used);
    a.max_relres = std::max(a.max_relres, b.max_relres);
    a.not_converged += b.not_converged;
    a.ms_spmm += b.ms_spmm;
    a.n_spmm += b.n_spmm;
    a.ms_precond += b.ms_precond;
    a.n_precond += b.n_precond;
    a.ms_loop += b.ms_loop;
    a.iters_run = std::max(a.iters_run, b.iters_run);
    a.refinements += b.refinements;
    a.fp64_rounds += b.fp64_rounds;
    a.ms_resid += b.ms_resid;
    a.n_resid += b.n_resid;
    a.diff_fused = a.diff_fused && b.diff_fused;
    // the same factor in every batch: its shapes as the last batch used them, measured if any batch measured
    a.ms_trsv_tune += b.ms_trsv_tune;
    a.trsv_shapes = a.trsv_shapes == SSP_TRSV_TUNED ? SSP_TRSV_TUNED : b.trsv_shapes;
    for (int i = 0; i < 3; i++) a.trsv_levels[i] = b.trsv_levels[i];
}

static void sparsify_impl(Context& C, const ssp_csc* graph, const ssp_params* prm, int32_t out_mem, ssp_csc_out* out,
                          ssp_stats* st, const ShardArgs* sh = nullptr) {
    SSP_REQUIRE(prm, SSP_ERR_INVALID, "params is NULL");
    SSP_REQUIRE(prm->epsilon > 0 && std::isfinite(prm->epsilon), SSP_ERR_INVALID, "epsilon must be positive");
    SSP_CUDA(cudaSetDevice(C.device));
    StageTimer T(C);
    T.mark();  // 0
    DevCsc g = to_device(C, graph, "in");
    DevGraph G;
    build_graph_from_csc(C, g.n, g.colptr, g.rowidx, g.val, g.nnz, G);
    T.mark();  // 1
    HostOutBuffers hob;
    if (out && out_mem == SSP_MEM_HOST && G.lap_nnz >= HOST_OUT_PREFAULT_MIN) hob.start(G.n, G.lap_nnz);
    const int64_t n = G.n;
    const int32_t k = jl_dim(prm, n);
    const double scale = jl_scale(prm, k);
    const bool finish_only = sh && sh->sq_in;
    int32_t col_lo = 0, kl = k;  // the global columns solved here
    const DevGraph& SG = (sh && sh->sketch_graph) ? *sh->sketch_graph : G;
    if (sh && sh->sq_out) {
        SSP_REQUIRE(sh->col_lo >= 0 && sh->col_lo < sh->col_hi && sh->col_hi <= k, SSP_ERR_INVALID,
                    "shard column range must satisfy 0 <= begin < end <= k");
        col_lo = sh->col_lo;
        kl = sh->col_hi - sh->col_lo;
    }
    // one shard of columns per call; otherwise all columns at once, or batches sized after the factorization
    const bool can_batch = !finish_only && !(sh && sh->sq_out);
    const int32_t forced = can_batch ? forced_batch(kl) : 0;
    const bool batched = can_batch && ((forced > 0 && forced < kl) || !columns_fit(C, G, kl, prm->precision));
    int32_t kb = kl;
    double* Y = nullptr;
    if (!finish_only && !batched) {
        Y = C.ws.get_t<double>("sp_Y", (size_t)n * tile_ld(kl));
        sketch_device(C, SG, kl, scale, prm->sketch_seed, prm->sketch_uniform, Y, tile_ld(kl), 1, col_lo);
    }
    T.mark();  // 2
    DevFactor F;
    FactorOptions fo;
    fo.seed = prm->factor_seed;
    fo.dense_threshold = prm->dense_threshold;
    fo.max_degree = prm->factor_max_degree;
    PcgOptions po;
    po.tol = prm->pcg_tol;
    po.abs_tol = prm->pcg_abs_tol;
    po.max_iters = prm->pcg_max_iters;
    po.verbose = prm->verbose;
    po.precision = prm->precision;
    double ms_tune = 0.0;
    int64_t deg_used = fo.max_degree;
    if (finish_only) {
        deg_used = 0;
    } else if (fo.max_degree < 0) {
        // the probe always uses global columns [0, min(k, SSP_PROBE_COLS)), so every rank of a split run picks
        // the same factor
        const double* probe = Y;
        const int32_t kp = std::min<int32_t>(k, SSP_PROBE_COLS);
        if (col_lo != 0 || kl < kp || batched) {
            double* Yp = C.ws.get_t<double>("sp_Yprobe", (size_t)n * tile_ld(kp));
            sketch_device(C, SG, kp, scale, prm->sketch_seed, prm->sketch_uniform, Yp, tile_ld(kp), 1, 0);
            probe = Yp;
        }
        deg_used = autotune_factor(C, n, G.lap_ptr, G.lap_idx, G.lap_val, 2 * G.m, G.max_deg, probe, kp, fo, po, F,
                                   &ms_tune);
    } else {
        factor_device(C, n, G.lap_ptr, G.lap_idx, G.lap_val, fo, F, "f");
    }
    T.mark();  // 3
    PcgReport rep;
    const double* Zt = nullptr;
    // the final product of the solve also forms the squared diff norms (sharded: this rank's share);
    // SSP_DIFF_FUSED=0 leaves them to the separate pass over the edges (the same sums, for comparison)
    const char* fe = getenv("SSP_DIFF_FUSED");
    const bool fuse = !(fe && fe[0] == '0');
    double* d2 = (finish_only || !fuse) ? nullptr
                 : (sh && sh->sq_out) ? sh->sq_out : C.ws.get_t<double>("sp_d2", G.m + 1);
    double* d2sum = batched ? C.ws.get_t<double>("sp_d2", G.m + 1) : nullptr;  // batches: their squared sums
    if (batched) {
        kb = forced > 0 ? forced : batch_after_factor(C, G, kl, prm->precision);
        Y = C.ws.get_t<double>("sp_Y", (size_t)n * tile_ld(kb));
        sketch_device(C, SG, kb, scale, prm->sketch_seed, prm->sketch_uniform, Y, tile_ld(kb), 1, 0);
    }
    if (!finish_only)
        pcg_device(C, n, G.lap_ptr, G.lap_idx, G.lap_val, F, Y, kb, &Zt, po, rep, nullptr, nullptr, G.lap_eid, d2);
    if (batched) {
        // the batches' squared diff norms accumulate tile by tile into d2sum: fused, they continue the single
        // pass's order exactly; from the separate pass, each batch's partial sum is added
        double* part = C.ws.get_t<double>("sp_d2part", G.m + 1);
        if (!rep.diff_fused) diff_sq_device(C, G.m, G.v1, G.v2, Zt, kb, n, d2sum);
        for (int32_t c0 = kb; c0 < kl; c0 += kb) {
            const int32_t kc = std::min(kb, kl - c0);
            sketch_device(C, SG, kc, scale, prm->sketch_seed, prm->sketch_uniform, Y, tile_ld(kc), 1, c0);
            PcgReport rb;
            pcg_device(C, n, G.lap_ptr, G.lap_idx, G.lap_val, F, Y, kc, &Zt, po, rb, nullptr, nullptr, G.lap_eid,
                       fuse ? d2sum : nullptr, true);
            if (!rb.diff_fused) {
                diff_sq_device(C, G.m, G.v1, G.v2, Zt, kc, n, part);
                add_device(C, G.m, part, d2sum);
            }
            merge_report(rep, rb, c0, kc);
        }
    }
    T.mark();  // 4
    if (sh && sh->sq_out) {
        if (!rep.diff_fused) diff_sq_device(C, G.m, G.v1, G.v2, Zt, kl, n, sh->sq_out);
        T.mark();  // 5
        SSP_CUDA(cudaStreamSynchronize(C.stream));
        if (st) {
            memset(st, 0, sizeof(*st));
            st->n = n;
            st->m_in = G.m;
            st->k = k;
            st->beta = beta_of(prm, n);
            st->nnz_factor = F.nnz;
            st->factor_levels = F.num_levels;
            st->pcg_max_iters_used = rep.max_iters_used;
            st->pcg_mean_iters = rep.mean_iters;
            st->pcg_max_relres = rep.max_relres;
            st->ms_assembly = T.ms(0, 1);
            st->ms_sketch = T.ms(1, 2);
            st->ms_factor = T.ms(2, 3);
            st->ms_solve = T.ms(3, 4);
            st->ms_leverage = T.ms(4, 5);
            st->ms_total = T.ms(0, 5);
            st->kernels_launched = C.kernels_launched;
            st->ms_spmm = rep.ms_spmm;
            st->n_spmm = rep.n_spmm;
            st->ms_precond = rep.ms_precond;
            st->n_precond = rep.n_precond;
            st->nnz_laplacian = G.lap_nnz;
            st->factor_max_degree_used = deg_used;
            st->ms_autotune = ms_tune;
            st->pcg_refinements = rep.refinements;
            st->pcg_fp64_rounds = rep.fp64_rounds;
            st->spmm_slabs = rep.spmm_slabs;
            copy_trsv_stats(*st, rep);
        }
        return;
    }
    double* d = C.ws.get_t<double>("sp_d", G.m + 1);
    double* p = C.ws.get_t<double>("sp_p", G.m + 1);
    double* coins = C.ws.get_t<double>("sp_coins", G.m + 1);
    if (finish_only)
        sqrt_device(C, G.m, sh->sq_in, d);
    else if (batched)
        sqrt_device(C, G.m, d2sum, d);
    else if (rep.diff_fused)
        sqrt_device(C, G.m, d2, d);
    else
        diff_norms_device(C, G.m, G.v1, G.v2, Zt, k, tile_ld(kl), d, n, true);
    const double beta = beta_of(prm, n);
    const double denom = prm->prob_variance_correction ? (double)k * scale * scale : (double)k;
    probs_device(C, G.m, G.w, d, beta, denom, p);
    T.mark();  // 5
    coins_device(C, G.m, prm->sampling_seed, coins);
    int64_t *lh_ptr;
    int32_t* lh_idx;
    double* lh_val;
    const int64_t nnz = sample_apply_device(C, G, p, coins, prm->reweight, &lh_ptr, &lh_idx, &lh_val, nullptr);
    int64_t* nd = C.ws.get_t<int64_t>("sp_ndiag", 1);
    SSP_CUDA(cudaMemsetAsync(nd, 0, sizeof(int64_t), C.stream));
    k_count_diag<<<grid_for(n, 256), 256, 0, C.stream>>>(n, lh_ptr, lh_idx, nd);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    T.mark();  // 6
    const int64_t ndiag = read_i64(C, nd);
    int64_t lg_diag = 0;
    {
        SSP_CUDA(cudaMemsetAsync(nd, 0, sizeof(int64_t), C.stream));
        k_count_diag<<<grid_for(n, 256), 256, 0, C.stream>>>(n, G.lap_ptr, G.lap_idx, nd);
        SSP_CHECK_LAUNCH();
        C.kernels_launched++;
        lg_diag = read_i64(C, nd);
    }
    if (out) {
        memset(out, 0, sizeof(*out));
        out->n = n;
        out->nnz = nnz;
        if (out_mem == SSP_MEM_DEVICE) {
            out->colptr = lh_ptr;
            out->rowidx = lh_idx;
            out->values = lh_val;
            out->mem = SSP_MEM_DEVICE;
            out->owned_by_context = 1;
        } else {
            hob.join();
            if (hob.colptr && hob.rowidx && hob.values && nnz <= hob.cap) {
                out->colptr = hob.colptr;
                out->rowidx = hob.rowidx;
                out->values = hob.values;
                hob.colptr = nullptr;
                hob.rowidx = nullptr;
                hob.values = nullptr;
            } else {
                out->colptr = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
                out->rowidx = (int32_t*)malloc(sizeof(int32_t) * (nnz + 1));
                out->values = (double*)malloc(sizeof(double) * (nnz + 1));
            }
            if (!out->colptr || !out->rowidx || !out->values) {
                free(out->colptr); free(out->rowidx); free(out->values);
                memset(out, 0, sizeof(*out));
                throw Error(SSP_ERR_NOMEM, "host allocation of the output failed");
            }
            copy_d2h(C, out->colptr, lh_ptr, sizeof(int64_t) * (n + 1));
            copy_d2h(C, out->rowidx, lh_idx, sizeof(int32_t) * nnz);
            copy_d2h(C, out->values, lh_val, sizeof(double) * nnz);
            out->mem = SSP_MEM_HOST;
        }
    }
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    if (st) {
        memset(st, 0, sizeof(*st));
        st->n = n;
        st->m_in = (G.lap_nnz - lg_diag) / 2;
        st->m_out = (nnz - ndiag) / 2;
        st->k = k;
        st->beta = beta;
        st->nnz_factor = F.nnz;
        st->factor_levels = F.num_levels;
        st->pcg_max_iters_used = rep.max_iters_used;
        st->pcg_mean_iters = rep.mean_iters;
        st->pcg_max_relres = rep.max_relres;
        st->ms_assembly = T.ms(0, 1);
        st->ms_sketch = T.ms(1, 2);
        st->ms_factor = T.ms(2, 3);
        st->ms_solve = T.ms(3, 4);
        st->ms_leverage = T.ms(4, 5);
        st->ms_sample = T.ms(5, 6);
        st->ms_total = T.ms(0, 6);
        st->kernels_launched = C.kernels_launched;
        st->ms_spmm = rep.ms_spmm;
        st->n_spmm = rep.n_spmm;
        st->ms_precond = rep.ms_precond;
        st->n_precond = rep.n_precond;
        st->nnz_laplacian = G.lap_nnz;
        st->factor_max_degree_used = deg_used;
        st->ms_autotune = ms_tune;
        st->pcg_refinements = rep.refinements;
        st->pcg_fp64_rounds = rep.fp64_rounds;
        st->spmm_slabs = rep.spmm_slabs;
        copy_trsv_stats(*st, rep);
    }
    if (prm->verbose) {
        fprintf(stderr, "[ssp] n=%lld m=%lld k=%d nnz(L)=%lld levels=%d (sparse %zu, dense %d, truncated %lld, compactions %d) "
                        "pcg iters max %d mean %.1f relres %.3g\n",
                (long long)n, (long long)G.m, k, (long long)F.nnz, F.num_levels, F.frontier_sizes.size(),
                F.dense_levels, (long long)F.truncated_rows, F.compactions, rep.max_iters_used, rep.mean_iters, rep.max_relres);
        fprintf(stderr, "[ssp] frontier sizes:");
        for (size_t i = 0; i < F.frontier_sizes.size(); i++)
            if (i < 24 || i % 50 == 0 || i + 5 > F.frontier_sizes.size())
                fprintf(stderr, " %zu:%lld", i, (long long)F.frontier_sizes[i]);
        fprintf(stderr, "\n");
    }
    if (prm->output_file && prm->output_file[0]) write_mtx_device(C, prm->output_file, n, lh_ptr, lh_idx, lh_val, "mtxw");
}

static void solve_impl(Context& C, const ssp_csc* lap, const double* Y, int32_t k, double* Z, int32_t mem,
                       const ssp_solve_opts* o, ssp_solve_report* rep, int32_t* iters, double* relres) {
    SSP_REQUIRE(lap && Y && Z && k > 0, SSP_ERR_INVALID, "solve: bad arguments");
    ssp_solve_opts od;
    ssp_solve_opts_default(&od);
    if (!o) o = &od;
    SSP_CUDA(cudaSetDevice(C.device));
    StageTimer T(C);
    T.mark();
    DevCsc L = to_device(C, lap, "lap");
    const int64_t n = L.n;
    const int64_t ld = tile_ld(k);
    const double* dY = Y;
    if (mem == SSP_MEM_HOST) {
        double* y = C.ws.get_t<double>("sl_Yrm", (size_t)n * k);
        SSP_CUDA(cudaMemcpyAsync(y, Y, sizeof(double) * n * k, cudaMemcpyHostToDevice, C.stream));
        dY = y;
    }
    double* Yt = C.ws.get_t<double>("sl_Yt", (size_t)n * ld);
    rowmajor_to_tiles(C, n, k, k, dY, Yt);
    DevFactor F;
    FactorOptions fo;
    fo.seed = o->factor_seed;
    fo.dense_threshold = o->dense_threshold;
    fo.max_degree = o->factor_max_degree;
    PcgOptions po;
    po.tol = o->tol;
    po.abs_tol = o->abs_tol;
    po.max_iters = o->max_iters;
    po.verbose = o->verbose;
    po.precision = o->precision;
    int64_t deg_used = fo.max_degree;
    if (fo.max_degree < 0) {
        const int64_t offdiag = L.nnz - n;  // every vertex of a connected Laplacian stores its diagonal
        deg_used = autotune_factor(C, n, L.colptr, L.rowidx, L.val, offdiag > 0 ? offdiag : L.nnz,
                                   max_offdiag_column(C, n, L.colptr, L.rowidx), Yt, k, fo, po, F, nullptr);
    } else {
        factor_device(C, n, L.colptr, L.rowidx, L.val, fo, F, "f");
    }
    T.mark();
    PcgReport pr;
    const double* Xt = nullptr;
    pcg_device(C, n, L.colptr, L.rowidx, L.val, F, Yt, k, &Xt, po, pr, iters, relres);
    T.mark();
    if (mem == SSP_MEM_HOST) {
        double* z = C.ws.get_t<double>("sl_Zrm", (size_t)n * k);
        tiles_to_rowmajor(C, n, k, Xt, z, k);
        SSP_CUDA(cudaMemcpyAsync(Z, z, sizeof(double) * n * k, cudaMemcpyDeviceToHost, C.stream));
    } else {
        tiles_to_rowmajor(C, n, k, Xt, Z, k);
    }
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    if (rep) {
        rep->k = k;
        rep->max_iters_used = pr.max_iters_used;
        rep->mean_iters = pr.mean_iters;
        rep->max_relres = pr.max_relres;
        rep->not_converged = pr.not_converged;
        rep->nnz_factor = F.nnz;
        rep->factor_levels = F.num_levels;
        rep->ms_factor = T.ms(0, 1);
        rep->ms_solve = T.ms(1, 2);
        rep->factor_max_degree_used = deg_used;
        rep->refinements = pr.refinements;
        rep->fp64_rounds = pr.fp64_rounds;
        rep->spmm_slabs = pr.spmm_slabs;
        copy_trsv_stats(*rep, pr);
    }
    if (pr.not_converged > 0)
        throw Error(SSP_ERR_NOT_CONVERGED, "solver did not converge: " + std::to_string(pr.not_converged) +
                                               " column(s) with relative residual >= 0.01 (max " +
                                               std::to_string(pr.max_relres) + ")");
}

template <class T>
static const T* stage_in(Context& C, const T* p, int64_t cnt, int32_t mem, const char* tag) {
    if (mem == SSP_MEM_DEVICE || cnt == 0) return p;
    T* d = C.ws.get_t<T>(tag, cnt);
    SSP_CUDA(cudaMemcpyAsync(d, p, sizeof(T) * cnt, cudaMemcpyHostToDevice, C.stream));
    return d;
}

// ---------------------------------------------------------------- several graphs at once
// The reference sparsifies one graph per process and solves its right-hand sides one after another
// (example.cc:551-568).  For many small graphs that leaves the GPU mostly idle, so a batch is run as the
// disjoint union of its graphs: one assembly, one factorization and one PCG for all of them.
//   * Graph b's vertices are [V_b, V_b + n_b) of the union and its edges [E_b, E_b + m_b) (the union's CSC
//     keeps each graph's columns together, and edges are extracted in CSC order).
//   * Its sketch uses its own seed, scale, k_b and edge ids counted from E_b; its factor draws are keyed by
//     in-graph vertex ids, and each graph is truncated by its own live-entry test at its own degree, so both
//     equal the lone run's.  A graph that asks for the autotuner (factor_max_degree = -1) gets the lone rule
//     graph by graph: the union is factored with every such graph at its light truncation, one 20-iteration
//     probe runs on the first columns with a residual history per graph, and the graphs predicted to need more
//     than 30 iterations are factored completely (the union is factored again).  There is no dense tail (it
//     looks at the whole Schur complement and would couple the graphs).
//   * The PCG keeps every scalar per (graph, column) (PcgSegments), so each graph's iterates are its own;
//     its reductions are blocked differently from a lone run's, so a served result equals the lone result
//     to the solve's rounding, not bit for bit.
//   * Probabilities and coins use each graph's beta, k, seeds and edge ids; L_H is assembled once and split.
__global__ void k_add_i64(int64_t count, int64_t* a, int64_t add) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        a[i] += add;
}
__global__ void k_add_i32(int64_t count, int32_t* a, int32_t add) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        a[i] += add;
}
// graph of every union vertex and the first vertex of that graph (V: nseg + 1 starts)
__global__ void k_vertex_graph(int64_t n, const int64_t* __restrict__ V, int32_t nseg, int32_t* __restrict__ rowseg,
                               int32_t* __restrict__ vbase) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        int32_t lo = 0, hi = nseg - 1;  // last s with V[s] <= v
        while (lo < hi) {
            const int32_t mid = (lo + hi + 1) >> 1;
            if (V[mid] <= v) lo = mid;
            else hi = mid - 1;
        }
        rowseg[v] = lo;
        vbase[v] = (int32_t)V[lo];
    }
}

static bool same_batch_options(const ssp_params& a, const ssp_params& b) {
    return a.factor_seed == b.factor_seed && a.precision == b.precision && a.pcg_tol == b.pcg_tol &&
           a.pcg_abs_tol == b.pcg_abs_tol && a.pcg_max_iters == b.pcg_max_iters && a.reweight == b.reweight &&
           a.dense_threshold == b.dense_threshold;
}

static void sparsify_batch_impl(Context& C, int32_t count, const ssp_csc* graphs, const ssp_params* prms,
                                ssp_csc_out* outs, ssp_stats* stats) {
    SSP_REQUIRE(count >= 1 && graphs && prms && outs, SSP_ERR_INVALID, "batch: need count >= 1, graphs, params, outs");
    for (int32_t b = 0; b < count; b++) memset(&outs[b], 0, sizeof(outs[b]));
    const ssp_params& p0 = prms[0];
    int64_t n = 0, nnz = 0;
    std::vector<int64_t> V(count + 1, 0), NZ(count + 1, 0), E(count + 1, 0);
    for (int32_t b = 0; b < count; b++) {
        const ssp_csc& g = graphs[b];
        const ssp_params& p = prms[b];
        SSP_REQUIRE(g.mem == SSP_MEM_HOST && g.n > 0 && g.nnz >= 0 && g.colptr && (g.nnz == 0 || (g.rowidx && g.values)),
                    SSP_ERR_INVALID, "batch: every graph must be a host CSC with n > 0");
        SSP_REQUIRE(g.colptr[0] == 0 && g.colptr[g.n] == g.nnz, SSP_ERR_INVALID, "batch: colptr must run 0 .. nnz");
        SSP_REQUIRE(p.epsilon > 0 && std::isfinite(p.epsilon), SSP_ERR_INVALID, "batch: epsilon must be positive");
        SSP_REQUIRE(same_batch_options(p, p0), SSP_ERR_INVALID,
                    "batch: factor seed, precision, PCG options and reweighting must agree");
        SSP_REQUIRE(p.dense_threshold == 0 && p.factor_max_degree >= -1, SSP_ERR_INVALID,
                    "batch: the graphs must ask for sparse-phase elimination (dense_threshold = 0, "
                    "factor_max_degree >= 0, or -1 for the autotuner)");
        // edges: upper entries with a non-zero value (sparsifier.rs:365), in CSC order
        int64_t m = 0;
        for (int64_t j = 0; j < g.n; j++)
            for (int64_t q = g.colptr[j]; q < g.colptr[j + 1]; q++) {
                SSP_REQUIRE(g.rowidx[q] >= 0 && g.rowidx[q] < g.n, SSP_ERR_INVALID, "batch: row index out of range");
                m += (g.rowidx[q] < j && g.values[q] != 0.0) ? 1 : 0;
            }
        V[b + 1] = V[b] + g.n;
        NZ[b + 1] = NZ[b] + g.nnz;
        E[b + 1] = E[b] + m;
    }
    n = V[count];
    nnz = NZ[count];
    SSP_REQUIRE(n < (int64_t)INT32_MAX, SSP_ERR_INVALID, "batch: the union must have fewer than 2^31 vertices");
    SSP_CUDA(cudaSetDevice(C.device));
    StageTimer T(C);
    T.mark();  // 0
    // the union CSC: each graph's arrays copied into place, then shifted by its vertex and entry offsets
    Workspace& W = C.ws;
    int64_t* ucp = W.get_t<int64_t>("bt_cp", n + 1);
    int32_t* uri = W.get_t<int32_t>("bt_ri", nnz + 1);
    double* uva = W.get_t<double>("bt_va", nnz + 1);
    for (int32_t b = 0; b < count; b++) {
        const ssp_csc& g = graphs[b];
        copy_h2d(C, ucp + V[b], g.colptr, sizeof(int64_t) * g.n);
        if (g.nnz) {
            copy_h2d(C, uri + NZ[b], g.rowidx, sizeof(int32_t) * g.nnz);
            copy_h2d(C, uva + NZ[b], g.values, sizeof(double) * g.nnz);
        }
        if (NZ[b]) k_add_i64<<<grid_for(g.n, 256), 256, 0, C.stream>>>(g.n, ucp + V[b], NZ[b]);
        if (V[b] && g.nnz) k_add_i32<<<grid_for(g.nnz, 256), 256, 0, C.stream>>>(g.nnz, uri + NZ[b], (int32_t)V[b]);
        SSP_CHECK_LAUNCH();
    }
    SSP_CUDA(cudaMemcpyAsync(ucp + n, &nnz, sizeof(int64_t), cudaMemcpyHostToDevice, C.stream));
    SSP_CUDA(cudaStreamSynchronize(C.stream));  // &nnz is a stack value
    DevGraph G;
    build_graph_from_csc(C, n, ucp, uri, uva, nnz, G, "bt_g");
    SSP_REQUIRE(G.m == E[count], SSP_ERR_INVALID, "batch: edge count of the union differs from its graphs'");
    int64_t* dV = W.get_t<int64_t>("bt_V", count + 1);
    int32_t* rowseg = W.get_t<int32_t>("bt_rowseg", n);
    int32_t* vbase = W.get_t<int32_t>("bt_vbase", n);
    SSP_CUDA(cudaMemcpyAsync(dV, V.data(), sizeof(int64_t) * (count + 1), cudaMemcpyHostToDevice, C.stream));
    k_vertex_graph<<<grid_for(n, 256), 256, 0, C.stream>>>(n, dV, count, rowseg, vbase);
    SSP_CHECK_LAUNCH();
    C.kernels_launched += 1 + 2 * count;
    T.mark();  // 1
    // sketch: graph b fills its rows' first k_b columns; the other columns of its rows stay zero
    std::vector<int32_t> k(count);
    int32_t kmax = 1;
    for (int32_t b = 0; b < count; b++) {
        k[b] = jl_dim(&prms[b], V[b + 1] - V[b]);
        kmax = std::max(kmax, k[b]);
    }
    const int64_t ld = tile_ld(kmax);
    double* Y = W.get_t<double>("bt_Y", (size_t)n * ld);
    SSP_CUDA(cudaMemsetAsync(Y, 0, sizeof(double) * (size_t)n * ld, C.stream));
    for (int32_t b = 0; b < count; b++)
        sketch_device_part(C, G, V[b], V[b + 1] - V[b], E[b], k[b], jl_scale(&prms[b], k[b]), prms[b].sketch_seed,
                           prms[b].sketch_uniform, Y, ld, 1, 0);
    T.mark();  // 2
    DevFactor F;
    FactorOptions fo;
    fo.seed = p0.factor_seed;
    fo.dense_threshold = 0;
    fo.max_degree = 0;
    fo.vbase = vbase;
    fo.vseg = rowseg;
    fo.seg_row0 = V;
    PcgOptions po;
    po.tol = p0.pcg_tol;
    po.abs_tol = p0.pcg_abs_tol;
    po.max_iters = p0.pcg_max_iters;
    po.verbose = p0.verbose;
    po.precision = p0.precision;
    // each graph's truncation: its own, or the autotuner's light degree to be probed
    std::vector<int64_t> maxdeg(count);
    bool tune = false;
    for (int32_t b = 0; b < count; b++) {
        tune = tune || prms[b].factor_max_degree < 0;
        maxdeg[b] = prms[b].factor_max_degree >= 0 ? prms[b].factor_max_degree
                                                    : autotune_light_degree(V[b + 1] - V[b], 2 * (E[b + 1] - E[b]));
    }
    fo.seg_max_degree = maxdeg;
    factor_device(C, n, G.lap_ptr, G.lap_idx, G.lap_val, fo, F, "bt_f");
    if (tune) {
        // the autotuner's probe, graph by graph (autotune_factor): 20 FP64 iterations on the first columns
        PcgOptions pp = po;
        pp.tol = 0.0;
        pp.abs_tol = 0.0;
        pp.max_iters = SSP_TUNE_PROBE_ITERS;
        pp.verbose = 0;
        pp.precision = SSP_PRECISION_FP64;
        PcgSegments ps;
        ps.row0 = V;
        ps.rowseg = rowseg;
        ps.record_history = true;
        int32_t kp = 1;
        for (int32_t b = 0; b < count; b++) {
            ps.k.push_back(std::min<int32_t>(k[b], SSP_PROBE_COLS));
            kp = std::max(kp, ps.k.back());
        }
        pp.segs = &ps;
        PcgReport pr;
        pcg_device(C, n, G.lap_ptr, G.lap_idx, G.lap_val, F, Y, kp, nullptr, pp, pr);
        // each graph's largest vertex degree, for the rule's hub test
        std::vector<int64_t> aptr(n + 1);
        copy_d2h(C, aptr.data(), G.adj_ptr, sizeof(int64_t) * (n + 1));
        bool again = false;
        for (int32_t b = 0; b < count; b++) {
            if (prms[b].factor_max_degree >= 0) continue;
            int64_t dmax = 0;
            for (int64_t v = V[b]; v < V[b + 1]; v++) dmax = std::max(dmax, aptr[v + 1] - aptr[v]);
            const std::vector<double> none;
            const double iters = autotune_predicted_iters(b < (int32_t)ps.history.size() ? ps.history[b] : none,
                                                          po.tol);
            if (!autotune_keep_light(iters, V[b + 1] - V[b], 2 * (E[b + 1] - E[b]), dmax)) {
                maxdeg[b] = 0;
                again = true;
            }
        }
        if (again) {
            fo.seg_max_degree = maxdeg;
            factor_device(C, n, G.lap_ptr, G.lap_idx, G.lap_val, fo, F, "bt_f");
        }
    }
    T.mark();  // 3
    PcgSegments segs;
    segs.row0 = V;
    segs.k = k;
    segs.rowseg = rowseg;
    po.segs = &segs;
    PcgReport rep;
    const double* Zt = nullptr;
    double* d2 = W.get_t<double>("bt_d2", G.m + 1);
    pcg_device(C, n, G.lap_ptr, G.lap_idx, G.lap_val, F, Y, kmax, &Zt, po, rep, nullptr, nullptr, G.lap_eid, d2);
    T.mark();  // 4
    double* d = W.get_t<double>("bt_d", G.m + 1);
    double* pr = W.get_t<double>("bt_p", G.m + 1);
    double* coins = W.get_t<double>("bt_coins", G.m + 1);
    // columns past a graph's k_b are zero in its rows, so they add nothing to its norms
    if (rep.diff_fused) sqrt_device(C, G.m, d2, d);
    else diff_norms_device(C, G.m, G.v1, G.v2, Zt, kmax, ld, d, n, true);
    for (int32_t b = 0; b < count; b++) {
        const int64_t mb = E[b + 1] - E[b], nb = V[b + 1] - V[b];
        const double scale = jl_scale(&prms[b], k[b]);
        const double denom = prms[b].prob_variance_correction ? (double)k[b] * scale * scale : (double)k[b];
        probs_device(C, mb, G.w + E[b], d + E[b], beta_of(&prms[b], nb), denom, pr + E[b]);
    }
    T.mark();  // 5
    for (int32_t b = 0; b < count; b++) coins_device(C, E[b + 1] - E[b], prms[b].sampling_seed, coins + E[b]);
    int64_t* lh_ptr;
    int32_t* lh_idx;
    double* lh_val;
    sample_apply_device(C, G, pr, coins, p0.reweight, &lh_ptr, &lh_idx, &lh_val, nullptr);
    T.mark();  // 6
    // split L_H: graph b's columns, its row ids shifted back
    std::vector<int64_t> hptr(n + 1);
    copy_d2h(C, hptr.data(), lh_ptr, sizeof(int64_t) * (n + 1));
    for (int32_t b = 0; b < count; b++) {
        const int64_t nb = V[b + 1] - V[b];
        const int64_t e0 = hptr[V[b]], e1 = hptr[V[b + 1]], cnt = e1 - e0;
        ssp_csc_out& o = outs[b];
        o.n = nb;
        o.nnz = cnt;
        o.mem = SSP_MEM_HOST;
        o.colptr = (int64_t*)malloc(sizeof(int64_t) * (nb + 1));
        o.rowidx = (int32_t*)malloc(sizeof(int32_t) * (cnt + 1));
        o.values = (double*)malloc(sizeof(double) * (cnt + 1));
        if (!o.colptr || !o.rowidx || !o.values) {
            for (int32_t a = 0; a <= b; a++) {
                free(outs[a].colptr); free(outs[a].rowidx); free(outs[a].values);
                memset(&outs[a], 0, sizeof(outs[a]));
            }
            throw Error(SSP_ERR_NOMEM, "host allocation of a batch output failed");
        }
        for (int64_t j = 0; j <= nb; j++) o.colptr[j] = hptr[V[b] + j] - e0;
        if (cnt) {
            copy_d2h(C, o.rowidx, lh_idx + e0, sizeof(int32_t) * cnt);
            copy_d2h(C, o.values, lh_val + e0, sizeof(double) * cnt);
        }
        for (int64_t q = 0; q < cnt; q++) o.rowidx[q] -= (int32_t)V[b];
    }
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    for (int32_t b = 0; b < count; b++) {
        const ssp_csc_out& o = outs[b];
        int64_t diag = 0;
        for (int64_t j = 0; j < o.n; j++)
            for (int64_t q = o.colptr[j]; q < o.colptr[j + 1]; q++) diag += o.rowidx[q] == j;
        int32_t it_max = 0;
        double it_sum = 0.0, rel_max = 0.0;
        for (int32_t j = 0; j < k[b]; j++) {
            const int64_t s = (int64_t)b * ld + j;
            it_max = std::max(it_max, segs.iters[s]);
            it_sum += segs.iters[s];
            rel_max = std::max(rel_max, segs.relres[s]);
        }
        if (stats) {
            ssp_stats& st = stats[b];
            memset(&st, 0, sizeof(st));
            st.n = o.n;
            st.m_in = E[b + 1] - E[b];
            st.m_out = (o.nnz - diag) / 2;
            st.k = k[b];
            st.beta = beta_of(&prms[b], o.n);
            st.pcg_max_iters_used = it_max;
            st.pcg_mean_iters = it_sum / k[b];
            st.pcg_max_relres = rel_max;
            // the batch's shared figures: every graph of the batch reports the same stage times and factor
            st.nnz_factor = F.nnz;
            st.factor_levels = F.num_levels;
            st.factor_max_degree_used = maxdeg[b];
            st.ms_assembly = T.ms(0, 1);
            st.ms_sketch = T.ms(1, 2);
            st.ms_factor = T.ms(2, 3);
            st.ms_solve = T.ms(3, 4);
            st.ms_leverage = T.ms(4, 5);
            st.ms_sample = T.ms(5, 6);
            st.ms_total = T.ms(0, 6);
            st.kernels_launched = C.kernels_launched;
            st.ms_spmm = rep.ms_spmm;
            st.n_spmm = rep.n_spmm;
            st.ms_precond = rep.ms_precond;
            st.n_precond = rep.n_precond;
            st.nnz_laplacian = G.lap_nnz;
            st.pcg_refinements = rep.refinements;
            st.pcg_fp64_rounds = rep.fp64_rounds;
            st.spmm_slabs = rep.spmm_slabs;
            copy_trsv_stats(st, rep);
        }
        if (prms[b].output_file && prms[b].output_file[0]) {
            std::string err;
            if (write_mtx(prms[b].output_file, o.n, o.colptr, o.rowidx, o.values, err) != SSP_OK)
                throw Error(SSP_ERR_IO, err);
        }
    }
}

}  // namespace ssp

using namespace ssp;

extern "C" {

const char* ssp_last_error(void) { return g_last_error.c_str(); }

int ssp_context_create(int32_t device, ssp_context** out) {
    return guarded([&] {
        SSP_REQUIRE(out, SSP_ERR_INVALID, "ctx out pointer is NULL");
        auto* c = new ssp_context();
        try {
            init_context(c->ctx, device);
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}

int ssp_context_destroy(ssp_context* c) {
    return guarded([&] {
        if (!c) return;
        destroy_context(c->ctx);
        delete c;
    });
}

int ssp_context_set_stream(ssp_context* c, void* stream) {
    return guarded([&] {
        SSP_REQUIRE(c, SSP_ERR_INVALID, "ctx is NULL");
        SSP_CUDA(cudaStreamSynchronize(c->ctx.stream));
        if (c->ctx.own_stream && c->ctx.stream && stream) {
            cudaStreamDestroy(c->ctx.stream);
            c->ctx.own_stream = false;
        }
        if (stream) {
            c->ctx.stream = (cudaStream_t)stream;
        } else if (!c->ctx.own_stream) {
            SSP_CUDA(cudaStreamCreateWithFlags(&c->ctx.stream, cudaStreamNonBlocking));
            c->ctx.own_stream = true;
        }
        // the old stream is idle (synchronized above), so its frees are done
        c->ctx.ws.set_stream(c->ctx.stream);
    });
}

int64_t ssp_context_kernels_launched(const ssp_context* c) { return c ? c->ctx.kernels_launched : 0; }
int64_t ssp_context_workspace_bytes(const ssp_context* c) { return c ? (int64_t)c->ctx.ws.total_bytes() : 0; }

void ssp_params_new(ssp_params* p, double epsilon, int32_t beta_constant, int32_t row_constant, int32_t verbose,
                    double jl_factor, double jl_scaling_factor, uint64_t sketch_seed, uint64_t sampling_seed,
                    int32_t bench, int32_t sketch_uniform, const char* output_file, int32_t streaming) {
    memset(p, 0, sizeof(*p));
    p->epsilon = epsilon;
    p->beta_constant = beta_constant;
    p->row_constant = row_constant;
    p->verbose = verbose;
    p->jl_factor = jl_factor;
    p->jl_scaling_factor = jl_scaling_factor;
    p->sketch_seed = sketch_seed;
    p->sampling_seed = sampling_seed;
    p->bench = bench;
    p->sketch_uniform = sketch_uniform;
    p->output_file = output_file;
    p->streaming = streaming;
    p->jl_dim_rule = SSP_JL_DIM_REF;
    p->jl_scale_rule = SSP_JL_SCALE_FIXED;
    p->prob_variance_correction = 0;
    p->reweight = SSP_REWEIGHT_INV_SQRT_P;
    p->pcg_tol = 0.0;
    p->pcg_abs_tol = std::sqrt(2e-7);
    p->pcg_max_iters = 400;
    p->factor_seed = 0;
    p->dense_threshold = 4096;
    p->factor_max_degree = -1;
    p->jl_dim_override = 0;
    p->precision = SSP_PRECISION_FP64;
}

void ssp_params_default(ssp_params* p) {
    ssp_params_new(p, 0.5, 4, 2, 0, 1.5, std::sqrt(3.0), 1, 1, 0, 1, "", 0);
}

void ssp_params_cli(ssp_params* p, double epsilon, int32_t verbose, uint64_t sketch_seed, uint64_t sampling_seed,
                    int32_t bench, const char* output_file) {
    ssp_params_new(p, epsilon, 4, 2, verbose, 4.0, std::sqrt(3.0), sketch_seed, sampling_seed, bench, 0, output_file,
                   0);
}

int32_t ssp_params_jl_dim(const ssp_params* p, int64_t n) { return jl_dim(p, n); }
double ssp_params_beta(const ssp_params* p, int64_t n) { return beta_of(p, n); }
double ssp_params_jl_scale(const ssp_params* p, int32_t k) { return jl_scale(p, k); }

void ssp_solve_opts_default(ssp_solve_opts* o) {
    o->tol = 0.0;
    o->abs_tol = std::sqrt(2e-7);
    o->max_iters = 400;
    o->factor_seed = 0;
    o->dense_threshold = 4096;
    o->verbose = 0;
    o->factor_max_degree = -1;
    o->precision = SSP_PRECISION_FP64;
}

int ssp_run_solve_lap(const double* shared_jl_cols, size_t num_rows, size_t num_cols, const int32_t* col_ptrs,
                      size_t col_ptrs_len, const int32_t* row_indices, const double* values, size_t nnz,
                      const char* solver_output_filename, int32_t num_nodes, int32_t verbose,
                      double* solution_out) {
    (void)solver_output_filename;
    return guarded([&] {
        std::lock_guard<std::mutex> lk(g_default_mu);
        SSP_REQUIRE(num_nodes > 0 && (size_t)num_nodes == num_rows && col_ptrs_len == (size_t)num_nodes + 1,
                    SSP_ERR_INVALID, "run_solve_lap: inconsistent dimensions");
        SSP_REQUIRE((size_t)col_ptrs[num_nodes] == nnz, SSP_ERR_INVALID, "run_solve_lap: col_ptrs[n] != nnz");
        Context& C = default_context();
        std::vector<int64_t> cp(num_nodes + 1);
        for (int32_t i = 0; i <= num_nodes; i++) cp[i] = col_ptrs[i];
        ssp_csc L{num_nodes, (int64_t)nnz, cp.data(), row_indices, values, SSP_MEM_HOST};
        ssp_solve_opts o;
        ssp_solve_opts_default(&o);
        o.verbose = verbose;
        solve_impl(C, &L, shared_jl_cols, (int32_t)num_cols, solution_out, SSP_MEM_HOST, &o, nullptr, nullptr,
                   nullptr);
    });
}

int ssp_solve_lap(ssp_context* c, const ssp_csc* lap, const double* Y, int32_t k, double* Z, int32_t mem,
                  const ssp_solve_opts* opts, ssp_solve_report* rep) {
    return guarded([&] {
        SSP_REQUIRE(c, SSP_ERR_INVALID, "ctx is NULL");
        solve_impl(c->ctx, lap, Y, k, Z, mem, opts, rep, nullptr, nullptr);
    });
}

int ssp_sparsify(ssp_context* c, const ssp_csc* graph, const ssp_params* params, int32_t out_mem, ssp_csc_out* out,
                 ssp_stats* stats) {
    return guarded([&] {
        SSP_REQUIRE(c, SSP_ERR_INVALID, "ctx is NULL");
        sparsify_impl(c->ctx, graph, params, out_mem, out, stats);
    });
}

int ssp_sparsify_batch(ssp_context* c, int32_t count, const ssp_csc* graphs, const ssp_params* params,
                       ssp_csc_out* outs, ssp_stats* stats) {
    return guarded([&] {
        SSP_REQUIRE(c, SSP_ERR_INVALID, "ctx is NULL");
        sparsify_batch_impl(c->ctx, count, graphs, params, outs, stats);
    });
}

static void host_out(const HostCsc& h, ssp_csc_out* out);

// the Laplacian's off-diagonal entries, negated, in their stored order (host arrays)
static void laplacian_to_graph_host(int64_t n, int64_t nnz, const int64_t* cp, const int32_t* ri, const double* va,
                                    HostCsc& g) {
    g.n = n;
    g.colptr.assign(n + 1, 0);
    g.rowidx.clear();
    g.val.clear();
    for (int64_t j = 0; j < n; j++) {
        SSP_REQUIRE(cp[j] <= cp[j + 1] && cp[j + 1] <= nnz, SSP_ERR_INVALID, "CSC colptr must be non-decreasing");
        for (int64_t p = cp[j]; p < cp[j + 1]; p++) {
            if (ri[p] == j) continue;
            g.rowidx.push_back(ri[p]);
            g.val.push_back(-va[p]);
        }
        g.colptr[j + 1] = (int64_t)g.rowidx.size();
    }
}

int ssp_laplacian_to_graph(const ssp_csc* lap, ssp_csc_out* graph) {
    return guarded([&] {
        SSP_REQUIRE(lap && graph && lap->mem == SSP_MEM_HOST, SSP_ERR_INVALID, "laplacian_to_graph needs a host CSC");
        SSP_REQUIRE(lap->n > 0 && lap->nnz >= 0 && lap->colptr && (lap->nnz == 0 || (lap->rowidx && lap->values)),
                    SSP_ERR_INVALID, "invalid CSC descriptor");
        SSP_REQUIRE(lap->colptr[0] == 0 && lap->colptr[lap->n] == lap->nnz, SSP_ERR_INVALID,
                    "CSC colptr must start at 0 and end at nnz");
        HostCsc g;
        laplacian_to_graph_host(lap->n, lap->nnz, lap->colptr, lap->rowidx, lap->values, g);
        host_out(g, graph);
    });
}

int ssp_sparsify_laplacian(ssp_context* c, const ssp_csc* lap, const ssp_params* params, int32_t out_mem,
                           ssp_csc_out* out, ssp_stats* stats) {
    return guarded([&] {
        SSP_REQUIRE(c, SSP_ERR_INVALID, "ctx is NULL");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        // on the device: the Laplacian (copied in when it is on the host), then its graph
        const DevCsc L = to_device(C, lap, "lapin");
        int64_t* gp = nullptr;
        int32_t* gi = nullptr;
        double* gv = nullptr;
        const int64_t gnnz = laplacian_to_graph_device(C, L.n, L.nnz, L.colptr, L.rowidx, L.val, &gp, &gi, &gv);
        const ssp_csc gc{L.n, gnnz, gp, gi, gv, SSP_MEM_DEVICE};
        sparsify_impl(C, &gc, params, out_mem, out, stats);
    });
}

int ssp_shard_leverage(ssp_context* c, const ssp_csc* graph, const ssp_params* params, int32_t col_begin,
                       int32_t col_end, double* sq, int64_t* m, ssp_stats* stats) {
    return guarded([&] {
        SSP_REQUIRE(c, SSP_ERR_INVALID, "ctx is NULL");
        Context& C = c->ctx;
        if (!sq) {
            SSP_REQUIRE(m, SSP_ERR_INVALID, "need sq or m");
            SSP_CUDA(cudaSetDevice(C.device));
            DevCsc g = to_device(C, graph, "in");
            DevGraph G;
            build_graph_from_csc(C, g.n, g.colptr, g.rowidx, g.val, g.nnz, G);
            SSP_CUDA(cudaStreamSynchronize(C.stream));
            *m = G.m;
            return;
        }
        ShardArgs sh;
        sh.col_lo = col_begin;
        sh.col_hi = col_end;
        sh.sq_out = sq;
        sparsify_impl(C, graph, params, SSP_MEM_DEVICE, nullptr, stats, &sh);
        if (m && stats) *m = stats->m_in;
    });
}

int ssp_sparsify_update(ssp_context* c, const ssp_csc* laplacian, const ssp_csc* new_edges, const ssp_params* params,
                        int32_t out_mem, ssp_csc_out* out, ssp_stats* stats) {
    return guarded([&] {
        SSP_REQUIRE(c && laplacian && new_edges, SSP_ERR_INVALID, "bad arguments");
        SSP_REQUIRE(laplacian->n == new_edges->n, SSP_ERR_INVALID, "the Laplacian and the new edges differ in size");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        DevCsc L = to_device(C, laplacian, "ul");
        DevCsc B = to_device(C, new_edges, "ub");
        DevGraph Gn;
        build_graph_from_csc(C, B.n, B.colptr, B.rowidx, B.val, B.nnz, Gn, "gn");
        int64_t* mp;
        int32_t* mi;
        double* mv;
        const int64_t mnnz =
            laplacian_plus_graph_device(C, L.n, L.colptr, L.rowidx, L.val, B.colptr, B.rowidx, B.val, &mp, &mi, &mv);
        ssp_csc merged;
        merged.n = L.n;
        merged.nnz = mnnz;
        merged.colptr = mp;
        merged.rowidx = mi;
        merged.values = mv;
        merged.mem = SSP_MEM_DEVICE;
        ShardArgs sh;
        sh.sketch_graph = &Gn;
        sparsify_impl(C, &merged, params, out_mem, out, stats, &sh);
    });
}

int ssp_shard_finish(ssp_context* c, const ssp_csc* graph, const ssp_params* params, const double* sq_total,
                     int32_t out_mem, ssp_csc_out* out, ssp_stats* stats) {
    return guarded([&] {
        SSP_REQUIRE(c && sq_total, SSP_ERR_INVALID, "ctx and sq_total are required");
        ShardArgs sh;
        sh.sq_in = sq_total;
        sparsify_impl(c->ctx, graph, params, out_mem, out, stats, &sh);
    });
}

// ---------------------------------------------------------------- a15: checks
int ssp_check_laplacian(ssp_context* c, const ssp_csc* lap, double tol, int64_t* bad_columns,
                        double* max_abs_colsum, int64_t* asymmetric_entries) {
    return guarded([&] {
        SSP_REQUIRE(c && bad_columns && max_abs_colsum && asymmetric_entries, SSP_ERR_INVALID, "bad arguments");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        DevCsc L = to_device(C, lap, "qc");
        laplacian_check_device(C, L.n, L.colptr, L.rowidx, L.val, tol, bad_columns, max_abs_colsum,
                               asymmetric_entries);
    });
}

int ssp_probe_vectors(ssp_context* c, int64_t n, int32_t p, uint64_t seed, int32_t mem, double* X) {
    return guarded([&] {
        SSP_REQUIRE(c && X && n > 0 && p > 0, SSP_ERR_INVALID, "bad arguments");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        double* d = mem == SSP_MEM_DEVICE ? X : C.ws.get_t<double>("q_X", (size_t)n * p);
        probe_vectors_device(C, n, p, seed, d);
        if (mem == SSP_MEM_HOST)
            SSP_CUDA(cudaMemcpyAsync(X, d, sizeof(double) * n * p, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
    });
}

int ssp_quadratic_forms(ssp_context* c, const ssp_csc* lap, const double* X, int32_t p, int32_t mem, double* out) {
    return guarded([&] {
        SSP_REQUIRE(c && X && out && p > 0, SSP_ERR_INVALID, "bad arguments");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        DevCsc L = to_device(C, lap, "qf");
        const double* dX = stage_in(C, X, L.n * (int64_t)p, mem, "qf_X");
        double* dout = mem == SSP_MEM_DEVICE ? out : C.ws.get_t<double>("qf_out", p);
        quadratic_forms_device(C, L.n, L.colptr, L.rowidx, L.val, dX, p, dout);
        if (mem == SSP_MEM_HOST)
            SSP_CUDA(cudaMemcpyAsync(out, dout, sizeof(double) * p, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
    });
}

int ssp_probe_quadratic_form(ssp_context* c, const ssp_csc* lap_g, const ssp_csc* lap_h, double epsilon,
                             int32_t probes, uint64_t seed, ssp_probe_result* res) {
    return guarded([&] {
        SSP_REQUIRE(c && lap_g && lap_h && res && probes > 0, SSP_ERR_INVALID, "bad arguments");
        SSP_REQUIRE(lap_g->n == lap_h->n, SSP_ERR_INVALID, "L_G and L_H must have the same size");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        const int64_t n = lap_g->n;
        double* X = C.ws.get_t<double>("q_X", (size_t)n * probes);
        double* q = C.ws.get_t<double>("q_forms", 2 * (size_t)probes);
        probe_vectors_device(C, n, probes, seed, X);
        DevCsc G = to_device(C, lap_g, "qg");
        quadratic_forms_device(C, n, G.colptr, G.rowidx, G.val, X, probes, q);
        DevCsc H = to_device(C, lap_h, "qh");
        quadratic_forms_device(C, n, H.colptr, H.rowidx, H.val, X, probes, q + probes);
        std::vector<double> h(2 * (size_t)probes);
        SSP_CUDA(cudaMemcpyAsync(h.data(), q, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
        // experiments.rs:95-121: non-strict bound tests, relative error against the graph's form
        memset(res, 0, sizeof(*res));
        res->probes = probes;
        std::vector<double> err(probes);
        for (int32_t j = 0; j < probes; j++) {
            const double og = h[j], sh = h[probes + j];
            if (sh >= og * (1.0 + epsilon)) res->upper_bound_violations++;
            if (sh <= og * (1.0 - epsilon)) res->lower_bound_violations++;
            err[j] = std::fabs(sh - og) / std::fabs(og);
        }
        double mean = 0.0, mx = err[0];
        for (double e : err) {
            mean += e;
            mx = std::max(mx, e);
        }
        mean /= probes;
        double var = 0.0;
        for (double e : err) var += (e - mean) * (e - mean);
        res->mean_relative_error = mean;
        res->std_dev_relative_error = std::sqrt(var / probes);
        res->max_relative_error = mx;
    });
}

int ssp_connected_components(ssp_context* c, const ssp_csc* m, int32_t mem, int32_t* labels, int64_t* count) {
    return guarded([&] {
        SSP_REQUIRE(c && count, SSP_ERR_INVALID, "bad arguments");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        DevCsc M = to_device(C, m, "cc");
        int32_t* d = (labels && mem == SSP_MEM_DEVICE) ? labels : C.ws.get_t<int32_t>("cc_labels", M.n);
        *count = components_device(C, M.n, M.colptr, M.rowidx, M.val, d);
        if (labels && mem == SSP_MEM_HOST) {
            SSP_CUDA(cudaMemcpyAsync(labels, d, sizeof(int32_t) * M.n, cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaStreamSynchronize(C.stream));
        }
    });
}

int ssp_csc_free(ssp_csc_out* out) {
    if (!out) return SSP_OK;
    if (out->mem == SSP_MEM_HOST) {
        free(out->colptr);
        free(out->rowidx);
        free(out->values);
    } else if (!out->owned_by_context) {
        cudaFree(out->colptr);
        cudaFree(out->rowidx);
        cudaFree(out->values);
    }
    memset(out, 0, sizeof(*out));
    return SSP_OK;
}

// a library-owned host CSC of n columns and nnz entries (freed with ssp_csc_free); nothing is left allocated
// when one of the three arrays cannot be
static void alloc_host_csc(ssp_csc_out* out, int64_t n, int64_t nnz) {
    memset(out, 0, sizeof(*out));
    int64_t* cp = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
    int32_t* ri = (int32_t*)malloc(sizeof(int32_t) * (nnz + 1));
    double* va = (double*)malloc(sizeof(double) * (nnz + 1));
    if (!cp || !ri || !va) {
        free(cp);
        free(ri);
        free(va);
        throw Error(SSP_ERR_NOMEM, "host allocation of the output failed");
    }
    out->n = n;
    out->nnz = nnz;
    out->colptr = cp;
    out->rowidx = ri;
    out->values = va;
    out->mem = SSP_MEM_HOST;
}

static void host_out(const HostCsc& h, ssp_csc_out* out) {
    alloc_host_csc(out, h.n, h.colptr.empty() ? 0 : h.colptr[h.n]);
    memcpy(out->colptr, h.colptr.data(), sizeof(int64_t) * (h.n + 1));
    if (out->nnz) {
        memcpy(out->rowidx, h.rowidx.data(), sizeof(int32_t) * out->nnz);
        memcpy(out->values, h.val.data(), sizeof(double) * out->nnz);
    }
}

int ssp_read_mtx(const char* path, ssp_csc_out* out) {
    return guarded([&] {
        SSP_REQUIRE(path && out, SSP_ERR_INVALID, "bad arguments");
        HostCsc h;
        std::string err;
        if (read_mtx(path, h, err) != 0) throw Error(SSP_ERR_IO, err);
        host_out(h, out);
    });
}

int ssp_write_mtx(const char* path, const ssp_csc* m) {
    return guarded([&] {
        SSP_REQUIRE(path && m && m->mem == SSP_MEM_HOST, SSP_ERR_INVALID, "write_mtx needs a host CSC");
        std::string err;
        if (write_mtx(path, m->n, m->colptr, m->rowidx, m->values, err) != 0) throw Error(SSP_ERR_IO, err);
    });
}

// the file parsed on the device when it can be (read_mtx_device), else by the host reader and copied up
static ssp_csc read_mtx_to_device(Context& C, const char* path, HostCsc& h) {
    int64_t n = 0, nnz = 0;
    int64_t* cp = nullptr;
    int32_t* ri = nullptr;
    double* va = nullptr;
    if (read_mtx_device(C, path, &n, &nnz, &cp, &ri, &va, "mtxr")) return ssp_csc{n, nnz, cp, ri, va, SSP_MEM_DEVICE};
    std::string err;
    if (read_mtx(path, h, err) != 0) throw Error(SSP_ERR_IO, err);
    return ssp_csc{h.n, h.colptr[h.n], h.colptr.data(), h.rowidx.data(), h.val.data(), SSP_MEM_HOST};
}

int ssp_sparsify_mtx(const char* input_file, const char* output_file, const ssp_params* params, ssp_stats* stats) {
    return guarded([&] {
        SSP_REQUIRE(input_file && params, SSP_ERR_INVALID, "bad arguments");
        // InputStream::new zeroes the stored diagonal (stream.rs:23-28): the edge extraction only
        // reads row < col, so the diagonal never reaches the sparsifier.
        ssp_params p = *params;
        p.output_file = output_file;
        std::lock_guard<std::mutex> lk(g_default_mu);
        Context& C = default_context();
        HostCsc h;
        const ssp_csc g = read_mtx_to_device(C, input_file, h);
        sparsify_impl(C, &g, &p, SSP_MEM_HOST, nullptr, stats);
    });
}

int ssp_read_mtx_device(ssp_context* ctx, const char* path, int32_t out_mem, ssp_csc_out* out) {
    return guarded([&] {
        SSP_REQUIRE(ctx && path && out, SSP_ERR_INVALID, "bad arguments");
        SSP_REQUIRE(out_mem == SSP_MEM_HOST || out_mem == SSP_MEM_DEVICE, SSP_ERR_INVALID, "bad out_mem");
        Context& C = ctx->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        HostCsc h;
        const ssp_csc g = read_mtx_to_device(C, path, h);
        if (g.mem == SSP_MEM_HOST && out_mem == SSP_MEM_HOST) {
            host_out(h, out);
            return;
        }
        memset(out, 0, sizeof(*out));
        out->n = g.n;
        out->nnz = g.nnz;
        if (out_mem == SSP_MEM_HOST) {
            alloc_host_csc(out, g.n, g.nnz);
            SSP_CUDA(cudaMemcpyAsync(out->colptr, g.colptr, sizeof(int64_t) * (g.n + 1), cudaMemcpyDeviceToHost,
                                     C.stream));
            SSP_CUDA(cudaMemcpyAsync(out->rowidx, g.rowidx, sizeof(int32_t) * g.nnz, cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaMemcpyAsync(out->values, g.values, sizeof(double) * g.nnz, cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaStreamSynchronize(C.stream));
            out->mem = SSP_MEM_HOST;
            return;
        }
        // device result in the context's buffers (a host-read file is copied into them)
        int64_t* cp = (int64_t*)C.ws.get("mtxr_colptr", sizeof(int64_t) * (g.n + 1));
        int32_t* ri = (int32_t*)C.ws.get("mtxr_rowidx", sizeof(int32_t) * (g.nnz + 1));
        double* va = (double*)C.ws.get("mtxr_val", sizeof(double) * (g.nnz + 1));
        if (g.mem == SSP_MEM_HOST) {
            SSP_CUDA(cudaMemcpyAsync(cp, g.colptr, sizeof(int64_t) * (g.n + 1), cudaMemcpyHostToDevice, C.stream));
            SSP_CUDA(cudaMemcpyAsync(ri, g.rowidx, sizeof(int32_t) * g.nnz, cudaMemcpyHostToDevice, C.stream));
            SSP_CUDA(cudaMemcpyAsync(va, g.values, sizeof(double) * g.nnz, cudaMemcpyHostToDevice, C.stream));
            SSP_CUDA(cudaStreamSynchronize(C.stream));
        }
        out->colptr = cp;
        out->rowidx = ri;
        out->values = va;
        out->mem = SSP_MEM_DEVICE;
        out->owned_by_context = 1;
    });
}

int ssp_write_mtx_device(ssp_context* ctx, const char* path, const ssp_csc* m) {
    return guarded([&] {
        SSP_REQUIRE(ctx && path && m, SSP_ERR_INVALID, "bad arguments");
        Context& C = ctx->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        const DevCsc d = to_device(C, m, "mtxw_in");
        write_mtx_device(C, path, d.n, d.colptr, d.rowidx, d.val, "mtxw");
    });
}

int ssp_parse_decimal(const char* s, size_t len, double* out) {
    if (!s || !out) return -1;
    return dec::parse_decimal(s, s + len, out);
}

int ssp_format_g17(double v, char* buf, size_t cap) {
    if (!buf || cap < 33) return -1;
    const int len = dec::format_g17(v, buf);
    if (len >= 0) buf[len] = 0;
    return len;
}

int ssp_gen_grid2d(int64_t nx, int64_t ny, double w, ssp_csc_out* out) {
    return guarded([&] {
        SSP_REQUIRE(nx > 0 && ny > 0 && out, SSP_ERR_INVALID, "bad arguments");
        HostCsc h;
        gen_grid2d(nx, ny, w, h);
        host_out(h, out);
    });
}
int ssp_gen_grid3d(int64_t nx, int64_t ny, int64_t nz, double lo, double hi, uint64_t seed, ssp_csc_out* out) {
    return guarded([&] {
        SSP_REQUIRE(nx > 0 && ny > 0 && nz > 0 && out, SSP_ERR_INVALID, "bad arguments");
        HostCsc h;
        gen_grid3d(nx, ny, nz, lo, hi, seed, h);
        host_out(h, out);
    });
}
int ssp_gen_er(int64_t n, double avg_degree, double wlo, double whi, uint64_t seed, ssp_csc_out* out) {
    return guarded([&] {
        SSP_REQUIRE(n > 1 && avg_degree > 0 && out, SSP_ERR_INVALID, "bad arguments");
        HostCsc h;
        gen_er(n, avg_degree, wlo, whi, seed, h);
        host_out(h, out);
    });
}
int ssp_edgelist_to_mtx(const char* input_path, const char* output_path, double default_weight) {
    return guarded([&] {
        SSP_REQUIRE(input_path && output_path, SSP_ERR_INVALID, "bad arguments");
        std::string err;
        if (edgelist_to_mtx(input_path, output_path, default_weight, err) != 0) throw Error(SSP_ERR_IO, err);
    });
}

int ssp_edgelist_to_mtx_device(ssp_context* c, const char* input_path, const char* output_path,
                               double default_weight, int32_t* on_device) {
    return guarded([&] {
        SSP_REQUIRE(c && input_path && output_path, SSP_ERR_INVALID, "bad arguments");
        SSP_CUDA(cudaSetDevice(c->ctx.device));
        if (on_device) *on_device = 0;
        if (edgelist_to_mtx_device(c->ctx, input_path, output_path, default_weight)) {
            if (on_device) *on_device = 1;
            return;
        }
        std::string err;
        if (edgelist_to_mtx(input_path, output_path, default_weight, err) != 0) throw Error(SSP_ERR_IO, err);
    });
}

int ssp_format_shortest(double v, char* buf, size_t cap) {
    if (!buf || cap < 2) return -1;
    const int len = dec::format_shortest_fixed(v, buf, (int)(cap - 1));
    if (len >= 0) buf[len] = 0;
    return len;
}

int ssp_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed, ssp_csc_out* out) {
    return guarded([&] {
        SSP_REQUIRE(scale >= 1 && scale <= 30 && edge_factor > 0 && a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0 &&
                        out,
                    SSP_ERR_INVALID, "bad arguments");
        HostCsc h;
        gen_rmat(scale, edge_factor, a, b, c, seed, h);
        host_out(h, out);
    });
}

int ssp_gen_rgg(int64_t n, double avg_degree, double wlo, double whi, uint64_t seed, ssp_csc_out* out) {
    return guarded([&] {
        SSP_REQUIRE(n > 1 && avg_degree > 0 && out, SSP_ERR_INVALID, "bad arguments");
        HostCsc h;
        gen_rgg(n, avg_degree, wlo, whi, seed, h);
        host_out(h, out);
    });
}

int ssp_context_release_workspace(ssp_context* c) {
    return guarded([&] {
        SSP_REQUIRE(c, SSP_ERR_INVALID, "ctx is NULL");
        SSP_CUDA(cudaSetDevice(c->ctx.device));
        SSP_CUDA(cudaStreamSynchronize(c->ctx.stream));
        c->ctx.ws.release();
        // the frees are stream-ordered: once they have run, the pool returns the memory to the device
        SSP_CUDA(cudaStreamSynchronize(c->ctx.stream));
    });
}

// ---------------------------------------------------------------- stage entry points
int ssp_stage_graph(ssp_context* c, const ssp_csc* graph, int64_t* m, int64_t* lap_nnz, int32_t* v1, int32_t* v2,
                    double* w, int64_t* lap_colptr, int32_t* lap_rowidx, double* lap_values) {
    return guarded([&] {
        SSP_REQUIRE(c && graph && m && lap_nnz, SSP_ERR_INVALID, "bad arguments");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        DevCsc g = to_device(C, graph, "in");
        DevGraph G;
        build_graph_from_csc(C, g.n, g.colptr, g.rowidx, g.val, g.nnz, G);
        *m = G.m;
        *lap_nnz = G.lap_nnz;
        if (v1) {
            if (G.m) {
                SSP_CUDA(cudaMemcpyAsync(v1, G.v1, sizeof(int32_t) * G.m, cudaMemcpyDeviceToHost, C.stream));
                SSP_CUDA(cudaMemcpyAsync(v2, G.v2, sizeof(int32_t) * G.m, cudaMemcpyDeviceToHost, C.stream));
                SSP_CUDA(cudaMemcpyAsync(w, G.w, sizeof(double) * G.m, cudaMemcpyDeviceToHost, C.stream));
            }
            SSP_CUDA(cudaMemcpyAsync(lap_colptr, G.lap_ptr, sizeof(int64_t) * (G.n + 1), cudaMemcpyDeviceToHost,
                                     C.stream));
            if (G.lap_nnz) {
                SSP_CUDA(cudaMemcpyAsync(lap_rowidx, G.lap_idx, sizeof(int32_t) * G.lap_nnz, cudaMemcpyDeviceToHost,
                                         C.stream));
                SSP_CUDA(cudaMemcpyAsync(lap_values, G.lap_val, sizeof(double) * G.lap_nnz, cudaMemcpyDeviceToHost,
                                         C.stream));
            }
        }
        SSP_CUDA(cudaStreamSynchronize(C.stream));
    });
}

int ssp_stage_sketch(ssp_context* c, int64_t n, int64_t m, const int32_t* v1, const int32_t* v2, const double* w,
                     int32_t mem, int32_t k, double scale, uint64_t seed, int32_t uniform, double* Y) {
    return guarded([&] {
        SSP_REQUIRE(c && n > 0 && m >= 0 && k > 0 && Y, SSP_ERR_INVALID, "bad arguments");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        DevGraph G;
        G.n = n;
        G.m = m;
        if (mem == SSP_MEM_HOST) {
            G.v1 = C.ws.get_t<int32_t>("g_v1", m + 1);
            G.v2 = C.ws.get_t<int32_t>("g_v2", m + 1);
            G.w = C.ws.get_t<double>("g_w", m + 1);
            SSP_CUDA(cudaMemcpyAsync(G.v1, v1, sizeof(int32_t) * m, cudaMemcpyHostToDevice, C.stream));
            SSP_CUDA(cudaMemcpyAsync(G.v2, v2, sizeof(int32_t) * m, cudaMemcpyHostToDevice, C.stream));
            SSP_CUDA(cudaMemcpyAsync(G.w, w, sizeof(double) * m, cudaMemcpyHostToDevice, C.stream));
        } else {
            G.v1 = (int32_t*)v1;
            G.v2 = (int32_t*)v2;
            G.w = (double*)w;
        }
        build_graph_from_edges(C, G);
        double* dY = Y;
        if (mem == SSP_MEM_HOST) dY = C.ws.get_t<double>("st_Y", (size_t)n * k);
        sketch_device(C, G, k, scale, seed, uniform, dY, k, 0);
        if (mem == SSP_MEM_HOST)
            SSP_CUDA(cudaMemcpyAsync(Y, dY, sizeof(double) * n * k, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
    });
}

int ssp_stage_factor(ssp_context* c, const ssp_csc* lap, uint64_t seed, int64_t dense_threshold,
                     int64_t max_degree, int64_t* nnz, int64_t* colptr, int32_t* rows, double* vals, double* D,
                     int32_t* level, int32_t* num_levels) {
    return guarded([&] {
        SSP_REQUIRE(c && lap && nnz, SSP_ERR_INVALID, "bad arguments");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        DevCsc L = to_device(C, lap, "lap");
        DevFactor F;
        FactorOptions fo;
        fo.seed = seed;
        fo.dense_threshold = dense_threshold;
        fo.max_degree = max_degree;
        factor_device(C, L.n, L.colptr, L.rowidx, L.val, fo, F, "f");
        *nnz = F.nnz;
        if (num_levels) *num_levels = F.num_levels;
        if (rows) {
            SSP_CUDA(cudaMemcpyAsync(colptr, F.col_ptr, sizeof(int64_t) * (L.n + 1), cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaMemcpyAsync(rows, F.col_idx, sizeof(int32_t) * F.nnz, cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaMemcpyAsync(vals, F.col_val, sizeof(double) * F.nnz, cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaMemcpyAsync(D, F.D, sizeof(double) * L.n, cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaMemcpyAsync(level, F.level, sizeof(int32_t) * L.n, cudaMemcpyDeviceToHost, C.stream));
        }
        SSP_CUDA(cudaStreamSynchronize(C.stream));
    });
}

int ssp_stage_precond(ssp_context* c, const ssp_csc* lap, uint64_t seed, int64_t dense_threshold,
                      int64_t max_degree, const double* R, int32_t k, double* Zout) {
    return guarded([&] {
        SSP_REQUIRE(c && lap && R && Zout && k > 0, SSP_ERR_INVALID, "bad arguments");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        DevCsc L = to_device(C, lap, "lap");
        DevFactor F;
        FactorOptions fo;
        fo.seed = seed;
        fo.dense_threshold = dense_threshold;
        fo.max_degree = max_degree;
        factor_device(C, L.n, L.colptr, L.rowidx, L.val, fo, F, "f");
        const int64_t ld = tile_ld(k);
        double* dR = C.ws.get_t<double>("pc_R", (size_t)L.n * ld);
        double* dZ = C.ws.get_t<double>("pc_Z", (size_t)L.n * ld);
        double* dRr = C.ws.get_t<double>("pc_Rrm", (size_t)L.n * k);
        SSP_CUDA(cudaMemcpyAsync(dRr, R, sizeof(double) * L.n * k, cudaMemcpyHostToDevice, C.stream));
        rowmajor_to_tiles(C, L.n, k, k, dRr, dR);
        precond_apply_device(C, F, dR, dZ, ld);
        tiles_to_rowmajor(C, L.n, k, dZ, dRr, k);
        SSP_CUDA(cudaMemcpyAsync(Zout, dRr, sizeof(double) * L.n * k, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
    });
}

int ssp_stage_diff_norms(ssp_context* c, int64_t n, int64_t m, const int32_t* v1, const int32_t* v2, const double* Z,
                         int32_t k, int32_t mem, double* d) {
    return guarded([&] {
        SSP_REQUIRE(c && k > 0 && n >= 0 && m >= 0 && (m == 0 || (v1 && v2 && Z && d)), SSP_ERR_INVALID,
                    "ssp_stage_diff_norms: need n >= 0, m >= 0, k > 0 and non-null arrays");
        if (mem == SSP_MEM_HOST)
            for (int64_t e = 0; e < m; e++)
                SSP_REQUIRE(v1[e] >= 0 && v1[e] < n && v2[e] >= 0 && v2[e] < n, SSP_ERR_INVALID,
                            "ssp_stage_diff_norms: edge " + std::to_string(e) + " has an endpoint outside [0, n)");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        if (m == 0) return;
        const int32_t* dv1 = stage_in(C, v1, m, mem, "dn_v1");
        const int32_t* dv2 = stage_in(C, v2, m, mem, "dn_v2");
        const double* dZ = stage_in(C, Z, n * (int64_t)k, mem, "dn_Z");
        double* dd = mem == SSP_MEM_DEVICE ? d : C.ws.get_t<double>("dn_d", m + 1);
        // device input is not checked on the host: an edge with an endpoint outside [0, n) gets d = NaN
        diff_norms_device(C, m, dv1, dv2, dZ, k, k, dd, n, false);
        if (mem == SSP_MEM_HOST && m)
            SSP_CUDA(cudaMemcpyAsync(d, dd, sizeof(double) * m, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
    });
}

int ssp_stage_probs(ssp_context* c, int64_t m, const double* w, const double* d, double beta, double denom,
                    int32_t mem, double* p) {
    return guarded([&] {
        SSP_REQUIRE(c && p, SSP_ERR_INVALID, "bad arguments");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        const double* dw = stage_in(C, w, m, mem, "pr_w");
        const double* dd = stage_in(C, d, m, mem, "pr_d");
        double* dp = mem == SSP_MEM_DEVICE ? p : C.ws.get_t<double>("pr_p", m + 1);
        probs_device(C, m, dw, dd, beta, denom, dp);
        if (mem == SSP_MEM_HOST && m)
            SSP_CUDA(cudaMemcpyAsync(p, dp, sizeof(double) * m, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
    });
}

int ssp_stage_coins(ssp_context* c, int64_t m, uint64_t seed, int32_t mem, double* coins) {
    return guarded([&] {
        SSP_REQUIRE(c && coins, SSP_ERR_INVALID, "bad arguments");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        double* dc = mem == SSP_MEM_DEVICE ? coins : C.ws.get_t<double>("co_c", m + 1);
        coins_device(C, m, seed, dc);
        if (mem == SSP_MEM_HOST && m)
            SSP_CUDA(cudaMemcpyAsync(coins, dc, sizeof(double) * m, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
    });
}

int ssp_stage_scan(ssp_context* c, const int32_t* in, int64_t n, int64_t* out) {
    return guarded([&] {
        SSP_REQUIRE(c && out && n >= 0 && (n == 0 || in), SSP_ERR_INVALID, "bad arguments");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        int32_t* di = C.ws.get_t<int32_t>("scan_in", n + 1);
        int64_t* dout = C.ws.get_t<int64_t>("scan_out", n + 1);
        if (n) SSP_CUDA(cudaMemcpyAsync(di, in, sizeof(int32_t) * n, cudaMemcpyHostToDevice, C.stream));
        exclusive_scan_i32_to_i64(C, di, dout, n, dout + n);
        SSP_CUDA(cudaMemcpyAsync(out, dout, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
    });
}

int ssp_stage_sample_apply(ssp_context* c, const ssp_csc* graph, const double* p, const double* coins,
                           int32_t reweight, int32_t mem, uint8_t* keep, ssp_csc_out* out) {
    return guarded([&] {
        SSP_REQUIRE(c && graph && p && coins && out, SSP_ERR_INVALID, "bad arguments");
        Context& C = c->ctx;
        SSP_CUDA(cudaSetDevice(C.device));
        DevCsc g = to_device(C, graph, "in");
        DevGraph G;
        build_graph_from_csc(C, g.n, g.colptr, g.rowidx, g.val, g.nnz, G);
        const double* dp = stage_in(C, p, G.m, mem, "sa_p");
        const double* dc = stage_in(C, coins, G.m, mem, "sa_c");
        uint8_t* dkeep = C.ws.get_t<uint8_t>("sa_keep", G.m + 1);
        int64_t* lp;
        int32_t* li;
        double* lv;
        int64_t nnz = sample_apply_device(C, G, dp, dc, reweight, &lp, &li, &lv, dkeep);
        alloc_host_csc(out, G.n, nnz);
        SSP_CUDA(cudaMemcpyAsync(out->colptr, lp, sizeof(int64_t) * (G.n + 1), cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaMemcpyAsync(out->rowidx, li, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaMemcpyAsync(out->values, lv, sizeof(double) * nnz, cudaMemcpyDeviceToHost, C.stream));
        if (keep && G.m)
            SSP_CUDA(cudaMemcpyAsync(keep, dkeep, G.m, mem == SSP_MEM_HOST ? cudaMemcpyDeviceToHost
                                                                            : cudaMemcpyDeviceToDevice,
                                     C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
    });
}

}  // extern "C"
