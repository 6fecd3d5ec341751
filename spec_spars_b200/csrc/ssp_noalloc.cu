// ssp_noalloc.cu -- the leverage-probability stage without any allocation.
//
// ssp_stage_leverage_probs_static computes, for every edge e = (v1_e, v2_e),
//     d_e = || Z[v1_e, :] - Z[v2_e, :] ||_2          (the per-edge effective-resistance estimate)
//     p_e = min(((beta * w_e) * d_e^2) / denom, 1)    (the sampling probability)
// with the same arithmetic, in the same order, as ssp_stage_diff_norms followed by ssp_stage_probs.
// The intermediate d lives in a file-scope device array instead of the context workspace, so the call
// needs no ssp_context and performs no cudaMalloc/cudaFree: it is meant for hosts whose device memory is
// owned by their own pool with a fixed budget, or that cannot accept the device-wide synchronisation a
// cudaFree implies, after start-up.
//
// Scratch contract:
//   * capacity SSP_STATIC_SCRATCH_EDGES doubles (8 MiB); larger m is rejected with SSP_ERR_CAPACITY
//     before anything is launched;
//   * nothing in the scratch has to start at zero: entries [0, m) are written before they are read;
//   * the scratch is shared by every call on a device, so two calls in flight at the same time on one
//     device (different streams or host threads) race -- callers serialise them (one stream, or events);
//   * the first call made with each device current loads this library's device code on that device (under
//     CUDA's lazy module loading that is when the scratch array itself is created, a device allocation) and
//     looks the scratch address up with cudaGetSymbolAddress; make that first call at start-up, before any
//     stream capture, so that no later call allocates;
//   * the address is kept per device index for the life of the process: after cudaDeviceReset (or anything
//     else that destroys the device's primary context) it is stale, so a process that resets a device must
//     not call this entry point on that device again.
#include <atomic>
#include <cstdio>

#include "ssp_internal.cuh"

namespace {

static __device__ __align__(256) double g_ssp_static_scratch[SSP_STATIC_SCRATCH_EDGES];

constexpr int kMaxDevices = 64;
std::atomic<double*> g_scratch_addr[kMaxDevices];

// d_e into the scratch: one warp per edge over row-major Z (leading dimension k), with the per-edge sum of
// k_diff_norms (warp_edge_sq: 32 columns at a time, a fixed xor butterfly, groups added in order).
// An edge with an endpoint outside [0, n) is not read and gets d_e = NaN, as in k_diff_norms.
__global__ void __launch_bounds__(256) k_norms_static(int64_t n, int64_t m, const int32_t* __restrict__ v1,
                                                      const int32_t* __restrict__ v2, const double* __restrict__ Z,
                                                      int32_t k, double* __restrict__ d) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t e = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < m; e += nw) {
        const int64_t a = v1[e], b = v2[e];
        if (a < 0 || a >= n || b < 0 || b >= n) {
            if (lane == 0) d[e] = __longlong_as_double(0x7ff8000000000000LL);
            continue;
        }
        const double acc = ssp::warp_edge_sq<false>(a, b, Z, k, k, n, lane);
        if (lane == 0) d[e] = sqrt(acc);
    }
}

// p_e from the scratch d_e with the body of k_probs (leverage_prob): a NaN ratio maps to probability 1.
__global__ void k_probs_static(int64_t m, const double* __restrict__ w, const double* __restrict__ d, double beta,
                               double denom, double* __restrict__ p) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x)
        p[e] = ssp::leverage_prob(w[e], d[e], beta, denom);
}

int fail(int code, const char* msg) {
    ssp::set_last_error(msg);
    return code;
}

}  // namespace

extern "C" int ssp_stage_leverage_probs_static(void* stream, int64_t n, int64_t m, const int32_t* v1,
                                               const int32_t* v2, const double* Z, int32_t k, const double* w,
                                               double beta, double denom, double* p) {
    char msg[192];
    if (m < 0 || n < 0 || k <= 0)
        return fail(SSP_ERR_INVALID, "ssp_stage_leverage_probs_static: need n >= 0, m >= 0, k > 0");
    if (m > (int64_t)SSP_STATIC_SCRATCH_EDGES) {
        snprintf(msg, sizeof msg,
                 "ssp_stage_leverage_probs_static: m = %lld edges exceeds the static scratch capacity of %lld edges",
                 (long long)m, (long long)SSP_STATIC_SCRATCH_EDGES);
        return fail(SSP_ERR_CAPACITY, msg);
    }
    if (m == 0) return SSP_OK;
    if (!v1 || !v2 || !Z || !w || !p)
        return fail(SSP_ERR_INVALID, "ssp_stage_leverage_probs_static: null device pointer");
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        snprintf(msg, sizeof msg, "ssp_stage_leverage_probs_static: cudaGetDevice: %s",
                 e != cudaSuccess ? cudaGetErrorString(e) : "device index out of range");
        return fail(e == cudaErrorNoDevice ? SSP_ERR_NO_DEVICE : SSP_ERR_CUDA, msg);
    }
    double* d = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!d) {
        void* addr = nullptr;
        e = cudaGetSymbolAddress(&addr, g_ssp_static_scratch);
        if (e != cudaSuccess || !addr) {
            snprintf(msg, sizeof msg, "ssp_stage_leverage_probs_static: cudaGetSymbolAddress: %s",
                     cudaGetErrorString(e));
            return fail(SSP_ERR_CUDA, msg);
        }
        d = static_cast<double*>(addr);
        g_scratch_addr[dev].store(d, std::memory_order_release);
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t warp_blocks = (m * 32 + 255) / 256;
    const int g1 = (int)(warp_blocks < 148 * 16 ? warp_blocks : 148 * 16);
    k_norms_static<<<g1, 256, 0, s>>>(n, m, v1, v2, Z, k, d);
    const int64_t blocks = (m + 255) / 256;
    const int g2 = (int)(blocks < 148 * 32 ? blocks : 148 * 32);
    k_probs_static<<<g2, 256, 0, s>>>(m, w, d, beta, denom, p);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(msg, sizeof msg, "ssp_stage_leverage_probs_static: launch: %s", cudaGetErrorString(e));
        return fail(SSP_ERR_CUDA, msg);
    }
    return SSP_OK;
}
