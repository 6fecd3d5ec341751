// ssp_quality.cu -- a15: checks of a Laplacian and of a sparsifier against its graph, on the device.
//
// Reference:
//   check_diagonal          sparsifier.rs:806-817  every column sums to 0 within 1e-10, the matrix is symmetric
//   compute_quadratic_form  sparsifier.rs:820-826  x^T L x
//   probe_quadratic_form    experiments.rs:88-122  uniform(-1, 1) probe vectors (tests.rs:50-59); a probe
//                                                 violates the bound when x^T L_H x >= (1 + eps) x^T L_G x
//                                                 or <= (1 - eps) x^T L_G x; relative errors |qH - qG| / |qG|
//   verify_ccs              experiments.rs:58-64   the sparsifier has as many connected components as the graph
// The probes here come from Philox (counter (vertex, probe), stream PROB) instead of thread_rng, so a check
// can be repeated exactly.
#include <cmath>

#include "ssp_internal.cuh"

namespace ssp {

namespace {

constexpr uint64_t STREAM_PROBE = 0x50524f42ull;  // "PROB"
constexpr int QF_WARPS = 8;                      // rows per block of the quadratic-form kernel

// one thread per column: the column's sum in storage order, and each entry's mirror found by binary search
// in the column of its row (rows sorted within a column); mismatched or missing mirrors are counted
__global__ void k_lap_check(int64_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                            const double* __restrict__ val, double tol, unsigned long long* __restrict__ bad_cols,
                            unsigned long long* __restrict__ max_abs_bits, unsigned long long* __restrict__ asym) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        unsigned long long miss = 0;
        for (int64_t t = ptr[j]; t < ptr[j + 1]; t++) {
            s += val[t];
            const int64_t i = idx[t];
            int64_t lo = ptr[i], hi = ptr[i + 1] - 1;
            bool found = false;
            while (lo <= hi) {
                const int64_t mid = (lo + hi) >> 1;
                const int32_t r = idx[mid];
                if (r == (int32_t)j) {
                    found = val[mid] == val[t];
                    break;
                }
                if (r < (int32_t)j) lo = mid + 1;
                else hi = mid - 1;
            }
            if (!found) miss++;
        }
        const double a = fabs(s);
        if (!(a <= tol)) atomicAdd(bad_cols, 1ull);
        atomicMax(max_abs_bits, (unsigned long long)__double_as_longlong(a));
        if (miss) atomicAdd(asym, miss);
    }
}

// probe vectors, column-major n x p: X[i + n j] = 2 u - 1, u = u53 of Philox((i, j), (seed, PROB)) word 0
__global__ void k_probe_vectors(int64_t n, int32_t p, uint64_t seed, double* __restrict__ X) {
    const int64_t total = n * (int64_t)p;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = t / n, i = t - j * n;
        const u64x4 r = philox((uint64_t)i, (uint64_t)j, 0, 0, seed, STREAM_PROBE);
        X[t] = 2.0 * ((double)(r.x >> 11) * 0x1.0p-53) - 1.0;
    }
}

// partial x_j^T L x_j over the rows of one block: warp per row gathers (L x_j)_i in a fixed lane order and a
// xor butterfly, then x_ij times it; the block adds its rows in warp order.  grid = (row blocks, p)
__global__ void __launch_bounds__(QF_WARPS * 32) k_quad_partial(int64_t n, const int64_t* __restrict__ ptr,
                                                                const int32_t* __restrict__ idx,
                                                                const double* __restrict__ val,
                                                                const double* __restrict__ X, int64_t rows_per_blk,
                                                                double* __restrict__ part) {
    __shared__ double s[QF_WARPS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t j = blockIdx.y;
    const double* x = X + j * n;
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_blk, r1 = min(n, r0 + rows_per_blk);
    double acc_w = 0.0;
    for (int64_t i = r0 + w; i < r1; i += QF_WARPS) {
        double a = 0.0;
        for (int64_t t = ptr[i] + lane; t < ptr[i + 1]; t += 32) a += val[t] * x[idx[t]];
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        acc_w += x[i] * a;
    }
    if (lane == 0) s[w] = acc_w;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tt = 0.0;
        for (int q = 0; q < QF_WARPS; q++) tt += s[q];
        part[j * gridDim.x + blockIdx.x] = tt;
    }
}

__global__ void k_quad_final(int32_t p, int nparts, const double* __restrict__ part, double* __restrict__ out) {
    for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < p; j += gridDim.x * blockDim.x) {
        double t = 0.0;
        for (int b = 0; b < nparts; b++) t += part[(int64_t)j * nparts + b];
        out[j] = t;
    }
}

// connected components: parent[v] <= v always holds, so every tree's root is its smallest vertex and the
// walk to it is finite
__device__ __forceinline__ int32_t cc_root(const int32_t* parent, int32_t v) {
    int32_t p = parent[v];
    while (p != v) {
        v = p;
        p = parent[v];
    }
    return v;
}

__global__ void k_cc_init(int64_t n, int32_t* __restrict__ parent) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        parent[v] = (int32_t)v;
}

// every off-diagonal nonzero joins the trees of its two vertices: the larger root hooks under the smaller
__global__ void k_cc_hook(int64_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                          const double* __restrict__ val, int32_t* parent, int32_t* __restrict__ changed) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        for (int64_t t = ptr[j]; t < ptr[j + 1]; t++) {
            const int32_t i = idx[t];
            if (i == (int32_t)j || val[t] == 0.0) continue;
            const int32_t a = cc_root(parent, i), b = cc_root(parent, (int32_t)j);
            if (a == b) continue;
            const int32_t hi = a > b ? a : b, lo = a > b ? b : a;
            atomicMin(&parent[hi], lo);
            *changed = 1;
        }
    }
}

__global__ void k_cc_compress(int64_t n, int32_t* parent, unsigned long long* __restrict__ roots) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r = cc_root(parent, (int32_t)v);
        parent[v] = r;
        if (r == (int32_t)v) atomicAdd(roots, 1ull);
    }
}

}  // namespace

void laplacian_check_device(Context& C, int64_t n, const int64_t* ptr, const int32_t* idx, const double* val,
                            double tol, int64_t* bad_cols, double* max_abs_colsum, int64_t* asym_entries) {
    unsigned long long* d = C.ws.get_t<unsigned long long>("q_check", 3);
    SSP_CUDA(cudaMemsetAsync(d, 0, 3 * sizeof(unsigned long long), C.stream));
    k_lap_check<<<grid_for(n, 256), 256, 0, C.stream>>>(n, ptr, idx, val, tol, d, d + 1, d + 2);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    unsigned long long h[3];
    SSP_CUDA(cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    *bad_cols = (int64_t)h[0];
    double m;
    memcpy(&m, &h[1], sizeof m);
    *max_abs_colsum = m;
    *asym_entries = (int64_t)h[2];
}

void probe_vectors_device(Context& C, int64_t n, int32_t p, uint64_t seed, double* X) {
    k_probe_vectors<<<grid_for(n * (int64_t)p, 256, 148 * 16), 256, 0, C.stream>>>(n, p, seed, X);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
}

void quadratic_forms_device(Context& C, int64_t n, const int64_t* ptr, const int32_t* idx, const double* val,
                            const double* X, int32_t p, double* out) {
    if (p <= 0) return;
    const int64_t rows_per_blk = std::max<int64_t>(QF_WARPS, ceil_div<int64_t>(n, 592));
    const int nparts = (int)ceil_div<int64_t>(n, rows_per_blk);
    double* part = C.ws.get_t<double>("q_part", (size_t)nparts * p);
    k_quad_partial<<<dim3((unsigned)nparts, (unsigned)p), QF_WARPS * 32, 0, C.stream>>>(n, ptr, idx, val, X,
                                                                                       rows_per_blk, part);
    k_quad_final<<<grid_for(p, 128), 128, 0, C.stream>>>(p, nparts, part, out);
    SSP_CHECK_LAUNCH();
    C.kernels_launched += 2;
}

int64_t components_device(Context& C, int64_t n, const int64_t* ptr, const int32_t* idx, const double* val,
                          int32_t* labels) {
    int32_t* changed = C.ws.get_t<int32_t>("q_cc_changed", 1);
    unsigned long long* roots = C.ws.get_t<unsigned long long>("q_cc_roots", 1);
    k_cc_init<<<grid_for(n, 256), 256, 0, C.stream>>>(n, labels);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    unsigned long long nroots = 0;
    // every round that hooks lowers some parent, so the loop ends; the cap only guards against a logic error
    const int max_rounds = 4096;
    for (int round = 0;; round++) {
        SSP_REQUIRE(round < max_rounds, SSP_ERR_CAPACITY, "connected components did not settle");
        SSP_CUDA(cudaMemsetAsync(changed, 0, sizeof(int32_t), C.stream));
        SSP_CUDA(cudaMemsetAsync(roots, 0, sizeof(unsigned long long), C.stream));
        k_cc_hook<<<grid_for(n, 256), 256, 0, C.stream>>>(n, ptr, idx, val, labels, changed);
        k_cc_compress<<<grid_for(n, 256), 256, 0, C.stream>>>(n, labels, roots);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += 2;
        int32_t h = 0;
        SSP_CUDA(cudaMemcpyAsync(&h, changed, sizeof h, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaMemcpyAsync(&nroots, roots, sizeof nroots, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
        if (!h) break;
    }
    return (int64_t)nroots;
}

}  // namespace ssp
