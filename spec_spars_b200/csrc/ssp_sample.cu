// ssp_sample.cu -- a9..a12: leverage estimates, probabilities, coins, reweighting and L_H.
//
// d_e = ||Z[v1] - Z[v2]||            compute_diff_norms   (sparsifier.rs:565-583)
// p_e = min(beta w d^2 / denom, 1)   compute_probs        (sparsifier.rs:542-562)
// keep iff coin_e < p_e              sample_and_reweight  (sparsifier.rs:635-680)
// L_H = L_G + dL, exact zeros drop   apply_reweightings   (sparsifier.rs:682-691)
//
// The diff-norm reduction order is fixed and mirrored by the CPU oracle, so given the same Z the norms are
// bit-identical: per 32-column tile, lane l squares the difference in its column (0 past k), an xor
// butterfly sums the 32 squares, and the tile sums are added in tile order.  The PCG's final product can
// form the same sums tile by tile while it gathers the same rows (pcg_device with an edge map).
#include "ssp_internal.cuh"

namespace ssp {

// ROOT = false leaves the sum of squares (one rank's share of the columns, summed across ranks later).
// An edge with an endpoint outside [0, n) is not read and gets NaN.
template <bool TM, bool ROOT = true>
__global__ void __launch_bounds__(256) k_diff_norms(int64_t m, const int32_t* __restrict__ v1,
                                                    const int32_t* __restrict__ v2, const double* __restrict__ Z,
                                                    int32_t k, int64_t ldz, int64_t n, double* __restrict__ d) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t e = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < m; e += nw) {
        const int64_t a = v1[e], b = v2[e];
        if (a < 0 || a >= n || b < 0 || b >= n) {
            if (lane == 0) d[e] = __longlong_as_double(0x7ff8000000000000LL);
            continue;
        }
        const double acc = warp_edge_sq<TM>(a, b, Z, k, ldz, n, lane);
        if (lane == 0) d[e] = ROOT ? sqrt(acc) : acc;
    }
}

__global__ void k_sqrt_vec(int64_t m, const double* __restrict__ sq, double* __restrict__ d) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x)
        d[e] = sqrt(sq[e]);
}

__global__ void k_probs(int64_t m, const double* __restrict__ w, const double* __restrict__ d, double beta,
                        double denom, double* __restrict__ p) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x)
        p[e] = leverage_prob(w[e], d[e], beta, denom);
}

__global__ void k_coins(int64_t m, uint64_t seed, double* __restrict__ coins) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x)
        coins[e] = edge_coin(seed, e);
}

// per edge: keep flag and the off-diagonal change X*-1 (Triplet::insert semantics)
__global__ void k_edge_changes(int64_t m, const double* __restrict__ w, const double* __restrict__ p,
                               const double* __restrict__ coins, int reweight, double* __restrict__ X,
                               uint8_t* __restrict__ keep) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x) {
        const bool kept = coins[e] < p[e];
        double x;
        if (kept) {
            const double t = reweight ? __ddiv_rn(w[e], p[e]) : __ddiv_rn(w[e], sqrt(p[e]));
            const double change = __dsub_rn(w[e], t);
            x = __dmul_rn(change, -1.0);
        } else {
            x = __dmul_rn(w[e], -1.0);
        }
        X[e] = x;
        if (keep) keep[e] = kept ? 1 : 0;
    }
}

// thread per vertex: diagonal change summed in edge order; then the L_H column, dropping exact zeros
__global__ void k_lh_count(int64_t n, const int64_t* __restrict__ adj_ptr, const int32_t* __restrict__ adj_nbr,
                           const int32_t* __restrict__ adj_eid, const double* __restrict__ X,
                           const int64_t* __restrict__ lg_ptr, const int32_t* __restrict__ lg_idx,
                           const double* __restrict__ lg_val, double* __restrict__ dchange,
                           int32_t* __restrict__ cnt) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        double dc = 0.0;
        for (int64_t p = adj_ptr[v]; p < adj_ptr[v + 1]; p++) dc = __dadd_rn(dc, X[adj_eid[p]]);
        dchange[v] = dc;
        int32_t c = 0;
        int64_t a = adj_ptr[v];
        for (int64_t t = lg_ptr[v]; t < lg_ptr[v + 1]; t++) {
            double x;
            if (lg_idx[t] == v) {
                x = __dadd_rn(lg_val[t], dc);
            } else {
                x = __dadd_rn(lg_val[t], __dmul_rn(X[adj_eid[a]], -1.0));
                a++;
            }
            c += (x != 0.0) ? 1 : 0;
        }
        cnt[v] = c;
    }
}

__global__ void k_lh_fill(int64_t n, const int64_t* __restrict__ adj_ptr, const int32_t* __restrict__ adj_eid,
                          const double* __restrict__ X, const int64_t* __restrict__ lg_ptr,
                          const int32_t* __restrict__ lg_idx, const double* __restrict__ lg_val,
                          const double* __restrict__ dchange, const int64_t* __restrict__ lh_ptr,
                          int32_t* __restrict__ lh_idx, double* __restrict__ lh_val) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        int64_t a = adj_ptr[v];
        int64_t q = lh_ptr[v];
        const double dc = dchange[v];
        for (int64_t t = lg_ptr[v]; t < lg_ptr[v + 1]; t++) {
            double x;
            if (lg_idx[t] == v) {
                x = __dadd_rn(lg_val[t], dc);
            } else {
                x = __dadd_rn(lg_val[t], __dmul_rn(X[adj_eid[a]], -1.0));
                a++;
            }
            if (x != 0.0) {
                lh_idx[q] = lg_idx[t];
                lh_val[q++] = x;
            }
        }
    }
}

void diff_norms_device(Context& C, int64_t m, const int32_t* v1, const int32_t* v2, const double* Z, int32_t k,
                       int64_t ldz, double* d, int64_t n, bool tile_major) {
    if (m == 0) return;
    if (tile_major)
        k_diff_norms<true><<<grid_for(m * 32, 256, 148 * 16), 256, 0, C.stream>>>(m, v1, v2, Z, k, ldz, n, d);
    else
        k_diff_norms<false><<<grid_for(m * 32, 256, 148 * 16), 256, 0, C.stream>>>(m, v1, v2, Z, k, ldz, n, d);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
}

void diff_sq_device(Context& C, int64_t m, const int32_t* v1, const int32_t* v2, const double* Z, int32_t k,
                    int64_t n_tile_major, double* sq) {
    if (m == 0) return;
    k_diff_norms<true, false><<<grid_for(m * 32, 256, 148 * 16), 256, 0, C.stream>>>(m, v1, v2, Z, k, k,
                                                                                     n_tile_major, sq);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
}

__global__ void k_add_vec(int64_t m, const double* __restrict__ src, double* __restrict__ dst) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x)
        dst[e] = __dadd_rn(dst[e], src[e]);
}

void add_device(Context& C, int64_t m, const double* src, double* dst) {
    if (m == 0) return;
    k_add_vec<<<grid_for(m, 256), 256, 0, C.stream>>>(m, src, dst);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
}

void sqrt_device(Context& C, int64_t m, const double* sq, double* d) {
    if (m == 0) return;
    k_sqrt_vec<<<grid_for(m, 256), 256, 0, C.stream>>>(m, sq, d);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
}

void probs_device(Context& C, int64_t m, const double* w, const double* d, double beta, double denom, double* p) {
    if (m == 0) return;
    k_probs<<<grid_for(m, 256), 256, 0, C.stream>>>(m, w, d, beta, denom, p);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
}

void coins_device(Context& C, int64_t m, uint64_t seed, double* coins) {
    if (m == 0) return;
    k_coins<<<grid_for(m, 256), 256, 0, C.stream>>>(m, seed, coins);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
}

int64_t sample_apply_device(Context& C, const DevGraph& G, const double* p, const double* coins, int reweight,
                            int64_t** lh_ptr_out, int32_t** lh_idx_out, double** lh_val_out, uint8_t* keep) {
    const int64_t n = G.n, m = G.m;
    Workspace& W = C.ws;
    double* X = W.get_t<double>("s_X", m + 1);
    double* dchange = W.get_t<double>("s_dchange", n + 1);
    int32_t* cnt = W.get_t<int32_t>("s_cnt", n + 1);
    int64_t* lh_ptr = W.get_t<int64_t>("s_lh_ptr", n + 1);
    int64_t* d_tot = W.get_t<int64_t>("s_tot", 1);
    if (m > 0) {
        k_edge_changes<<<grid_for(m, 256), 256, 0, C.stream>>>(m, G.w, p, coins, reweight, X, keep);
        SSP_CHECK_LAUNCH();
        C.kernels_launched++;
    }
    k_lh_count<<<grid_for(n, 128), 128, 0, C.stream>>>(n, G.adj_ptr, G.adj_nbr, G.adj_eid, X, G.lap_ptr, G.lap_idx,
                                                       G.lap_val, dchange, cnt);
    SSP_CHECK_LAUNCH();
    SSP_CUDA(cudaMemsetAsync(cnt + n, 0, sizeof(int32_t), C.stream));
    exclusive_scan_i32_to_i64(C, cnt, lh_ptr, n + 1, d_tot);
    int64_t nnz = read_i64(C, d_tot);
    int32_t* lh_idx = W.get_t<int32_t>("s_lh_idx", nnz + 1);
    double* lh_val = W.get_t<double>("s_lh_val", nnz + 1);
    k_lh_fill<<<grid_for(n, 128), 128, 0, C.stream>>>(n, G.adj_ptr, G.adj_eid, X, G.lap_ptr, G.lap_idx, G.lap_val,
                                                      dchange, lh_ptr, lh_idx, lh_val);
    SSP_CHECK_LAUNCH();
    C.kernels_launched += 2;
    *lh_ptr_out = lh_ptr;
    *lh_idx_out = lh_idx;
    *lh_val_out = lh_val;
    return nnz;
}

}  // namespace ssp
