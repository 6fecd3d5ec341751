// ssp_autotune.cu -- chooses how far the approximate Cholesky elimination should go.
//
// The reference always eliminates every vertex (example.cc:332-471).  That is the right preconditioner
// for ill-conditioned meshes, but on expander-like graphs the Schur complement densifies quickly, the
// factor grows to several times the graph, and PCG converges almost as fast with the diagonal of an
// early Schur complement -- while every PCG iteration pays gathers proportional to nnz(A) + 2 nnz(L).
//
// Rule: factor with the lightest truncation (stop once the Schur complement's average degree exceeds
// 1.05 d0 + 1, d0 the graph's average degree), run a 20-iteration PCG probe on the first SSP_PROBE_COLS
// columns of the actual right-hand sides, and estimate the iterations to reach the tolerance from the contraction
// rate of the last ten probe iterations.  A graph whose lightly preconditioned system converges within
// 30 iterations keeps that factor, and so does one with power-law hubs (largest vertex degree at least 16 times
// the average) that converges within 150: there complete elimination builds factors with thousands of
// latency-bound levels (R-MAT scale 18, measured on B200: 7,107 levels, 1.46 s per preconditioner application
// and 84 s per sparsification, against 4.9 ms and 4.0 s for the light factor at 56 instead of 54 iterations).
// Otherwise the elimination runs to completion.  Both factorizations, and so the choice, are deterministic.
#include <cmath>
#include <vector>

#include "ssp_internal.cuh"

namespace ssp {

constexpr int TUNE_PROBE_ITERS = SSP_TUNE_PROBE_ITERS;
constexpr double TUNE_MAX_ITERS = SSP_TUNE_MAX_ITERS;
constexpr double TUNE_MAX_ITERS_SKEWED = 150.0;
constexpr double TUNE_SKEW = 16.0;

bool autotune_keep_light(double predicted_iters, int64_t n, int64_t lap_offdiag_nnz, int64_t max_vertex_degree) {
    if (predicted_iters <= TUNE_MAX_ITERS) return true;
    const double d0 = n > 0 ? (double)lap_offdiag_nnz / (double)n : 0.0;
    return predicted_iters <= TUNE_MAX_ITERS_SKEWED && d0 > 0 && (double)max_vertex_degree >= TUNE_SKEW * d0;
}

int64_t autotune_light_degree(int64_t n, int64_t lap_offdiag_nnz) {
    const double d0 = n > 0 ? (double)lap_offdiag_nnz / (double)n : 0.0;
    return (int64_t)std::ceil(1.05 * d0) + 1;
}

double autotune_predicted_iters(const std::vector<double>& hist, double tol) {
    const double tol_rel = tol > 0 ? tol : 1e-6;
    double iters = 1e9;
    const size_t h = hist.size();
    if (h >= 2 && hist.back() <= tol_rel) {
        iters = (double)h;  // converged within the probe
    } else if (h >= 4) {
        const size_t a = h / 2;
        const double r0 = hist[a - 1], r1 = hist[h - 1];
        if (r0 > 0 && r1 > 0 && r1 < r0) {
            const double rho = std::pow(r1 / r0, 1.0 / (double)(h - a));
            iters = (double)h + std::log(tol_rel / r1) / std::log(rho);
        }
    }
    return iters;
}

int64_t autotune_factor(Context& C, int64_t n, const int64_t* lap_ptr, const int32_t* lap_idx, const double* lap_val,
                        int64_t lap_offdiag_nnz, int64_t max_vertex_degree, const double* Ytiles, int32_t k,
                        const FactorOptions& base, const PcgOptions& popt, DevFactor& F, double* ms_tuning) {
    const int64_t light = autotune_light_degree(n, lap_offdiag_nnz);
    cudaEvent_t e0, e1;
    SSP_CUDA(cudaEventCreate(&e0));
    SSP_CUDA(cudaEventCreate(&e1));
    SSP_CUDA(cudaEventRecord(e0, C.stream));
    FactorOptions fo = base;
    fo.max_degree = light;
    factor_device(C, n, lap_ptr, lap_idx, lap_val, fo, F, "f");
    PcgOptions po = popt;
    po.tol = 0.0;
    po.abs_tol = 0.0;
    po.max_iters = TUNE_PROBE_ITERS;
    po.verbose = 0;
    po.precision = SSP_PRECISION_FP64;  // the choice must not depend on the solve's precision
    std::vector<double> hist;
    po.history = &hist;
    PcgReport rep;
    const int32_t kp = std::min<int32_t>(k, SSP_PROBE_COLS);
    pcg_device(C, n, lap_ptr, lap_idx, lap_val, F, Ytiles, kp, nullptr, po, rep);
    const double iters = autotune_predicted_iters(hist, popt.tol);
    int64_t chosen = light;
    if (!autotune_keep_light(iters, n, lap_offdiag_nnz, max_vertex_degree)) {
        chosen = 0;
        fo.max_degree = 0;
        factor_device(C, n, lap_ptr, lap_idx, lap_val, fo, F, "f");
    }
    if (popt.verbose)
        fprintf(stderr, "[ssp] autotune: truncation at degree %lld predicts %.1f PCG iterations -> %s\n",
                (long long)light, iters, chosen ? "truncated factor" : "complete elimination");
    SSP_CUDA(cudaEventRecord(e1, C.stream));
    SSP_CUDA(cudaEventSynchronize(e1));
    float tt = 0;
    SSP_CUDA(cudaEventElapsedTime(&tt, e0, e1));
    if (ms_tuning) *ms_tuning = tt;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return chosen;
}

}  // namespace ssp
