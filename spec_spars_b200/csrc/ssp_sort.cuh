// ssp_sort.cuh -- bitonic sorting networks (warp registers and block shared/global memory).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ssp {

// Ascending bitonic sort of one (key, value) per lane across a full warp.
// Equal keys never swap, so a pair with equal keys keeps both entries.
template <class K, class V, class Less>
__device__ __forceinline__ void warp_bitonic_kv(K& key, V& val, int lane, Less less) {
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            K ok = __shfl_xor_sync(0xffffffffu, key, stride);
            V ov = __shfl_xor_sync(0xffffffffu, val, stride);
            bool up = (lane & size) == 0;
            bool lower = (lane & stride) == 0;
            bool take = lower ? (up ? less(ok, key) : less(key, ok)) : (up ? less(key, ok) : less(ok, key));
            if (take) {
                key = ok;
                val = ov;
            }
        }
    }
}

// Block-wide ascending bitonic sort of P (power of two) slots; P >= 2.
template <bool PAIRS, class K, class V, class Less>
__device__ void block_bitonic_kv(K* keys, V* vals, int P, Less less) {
    for (int size = 2; size <= P; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < (P >> 1); i += blockDim.x) {
                int lo = 2 * stride * (i / stride) + (i % stride);
                int hi = lo + stride;
                bool up = (lo & size) == 0;
                K a = keys[lo], b = keys[hi];
                bool swap = up ? less(b, a) : less(a, b);
                if (swap) {
                    keys[lo] = b;
                    keys[hi] = a;
                    if (PAIRS) {
                        V t = vals[lo];
                        vals[lo] = vals[hi];
                        vals[hi] = t;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Entries of the factorization: (row u, weight w) with two orders.
struct EntUW {  // (u asc, w asc)
    __device__ __forceinline__ bool operator()(int32_t ua, double wa, int32_t ub, double wb) const {
        return ua != ub ? ua < ub : wa < wb;
    }
};
struct EntWU {  // (w asc, u asc)
    __device__ __forceinline__ bool operator()(int32_t ua, double wa, int32_t ub, double wb) const {
        return wa != wb ? wa < wb : ua < ub;
    }
};

template <class Less>
__device__ __forceinline__ void warp_bitonic_ent(int32_t& u, double& w, int lane, Less less) {
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            int32_t ou = __shfl_xor_sync(0xffffffffu, u, stride);
            double ow = __shfl_xor_sync(0xffffffffu, w, stride);
            bool up = (lane & size) == 0;
            bool lower = (lane & stride) == 0;
            bool take = lower ? (up ? less(ou, ow, u, w) : less(u, w, ou, ow))
                              : (up ? less(u, w, ou, ow) : less(ou, ow, u, w));
            if (take) {
                u = ou;
                w = ow;
            }
        }
    }
}

template <class Less>
__device__ void block_bitonic_ent(int32_t* us, double* ws, int P, Less less) {
    for (int size = 2; size <= P; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < (P >> 1); i += blockDim.x) {
                int lo = 2 * stride * (i / stride) + (i % stride);
                int hi = lo + stride;
                bool up = (lo & size) == 0;
                int32_t ua = us[lo], ub = us[hi];
                double wa = ws[lo], wb = ws[hi];
                bool swap = up ? less(ub, wb, ua, wa) : less(ua, wa, ub, wb);
                if (swap) {
                    us[lo] = ub; us[hi] = ua;
                    ws[lo] = wb; ws[hi] = wa;
                }
            }
            __syncthreads();
        }
    }
}

}  // namespace ssp
