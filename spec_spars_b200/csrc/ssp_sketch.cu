// ssp_sketch.cu -- a4: Y = B^T Q with Q generated in registers from Philox.
//
// Reference: jl_sketch_colwise / populate_row / hash_with_inputs (sparsifier.rs:379-539).
// Y[v, j] = sum over edges e incident to v, in edge order, of (h(e,j) * scale) * b_ev with
// b_ev = -sqrt(w_e) at the smaller endpoint and +sqrt(w_e) at the larger (sparsifier.rs:97-109).
// Each product and each addition rounds separately (the reference multiplies the row by the
// value, then adds it), so the result is bit-identical to the oracle.
//
// One warp per (vertex, 256-column tile).  Lane l owns columns tile*256 + l + 32 t (t < 8), so
// every store instruction writes 32 consecutive doubles.  The 256 sign bits of one edge come from
// one Philox4x64 call; up to 32 edges are hashed at once (one per lane) and their words are
// broadcast with shuffles.  The output is row-major (leading dimension ldy) or tile-major (the
// PCG layout, see tile_off).  A block may hold a range [col_lo, col_lo + k) of the global columns (one
// rank's share when the columns are split across GPUs): every entry depends on its global column only.
#include "ssp_internal.cuh"

namespace ssp {

__global__ void __launch_bounds__(256) k_sketch_sign(int64_t n, int64_t v0, int64_t e0, int64_t nrows,
                                                     const int64_t* __restrict__ adj_ptr,
                                                     const int32_t* __restrict__ adj_eid,
                                                     const int32_t* __restrict__ v2, const double* __restrict__ w,
                                                     int32_t col_lo, int32_t col_hi, int32_t tile_lo,
                                                     int32_t ntiles, double scale, uint64_t seed,
                                                     double* __restrict__ Y, int64_t ldy, int tm) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t item = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; item < n * ntiles; item += nw) {
        const int64_t v = v0 + item / ntiles;
        const int32_t tile = tile_lo + (int32_t)(item - (v - v0) * ntiles);
        double acc[8];
#pragma unroll
        for (int t = 0; t < 8; t++) acc[t] = 0.0;
        const int64_t s = adj_ptr[v], e_end = adj_ptr[v + 1];
        for (int64_t p0 = s; p0 < e_end; p0 += 32) {
            const int cnt = (e_end - p0) < 32 ? (int)(e_end - p0) : 32;
            uint64_t r0 = 0, r1 = 0, r2 = 0, r3 = 0;
            double b = 0.0;
            if (lane < cnt) {
                int32_t e = adj_eid[p0 + lane];
                u64x4 r = philox((uint64_t)(e - e0), (uint64_t)tile, 0, 0, seed, STREAM_SIGN);
                r0 = r.x; r1 = r.y; r2 = r.z; r3 = r.w;
                double sw = sqrt(w[e]);
                b = (v2[e] == (int32_t)v) ? sw : -sw;
            }
            for (int i = 0; i < cnt; i++) {
                const uint64_t q0 = __shfl_sync(0xffffffffu, r0, i);
                const uint64_t q1 = __shfl_sync(0xffffffffu, r1, i);
                const uint64_t q2 = __shfl_sync(0xffffffffu, r2, i);
                const uint64_t q3 = __shfl_sync(0xffffffffu, r3, i);
                const double bi = __shfl_sync(0xffffffffu, b, i);
                // (+-scale) * b_ev is +-(scale * b_ev) exactly (negation is exact): one product per edge
                const double sb = __dmul_rn(scale, bi);
                const uint64_t words[4] = {q0, q1, q2, q3};
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    // column c = lane + 32 t inside the tile: word t>>1, bit lane + 32 (t & 1)
                    const uint64_t bit = (words[t >> 1] >> (lane + 32 * (t & 1))) & 1ull;
                    acc[t] = __dadd_rn(acc[t], bit ? -sb : sb);
                }
            }
        }
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const int64_t col = (int64_t)tile * 256 + lane + 32 * t;
            if (col >= col_lo && col < col_hi) {
                const int64_t lc = col - col_lo;  // column of the stored block
                Y[tm ? tile_off(nrows, v, lc) : v * ldy + lc] = acc[t];
            }
        }
    }
}

// Uniform (-1,1) entries: 32 bits each, 8 per Philox call (hash_with_inputs_alt, sparsifier.rs:410-420).
__global__ void __launch_bounds__(256) k_sketch_unif(int64_t n, int64_t v0, int64_t e0, int64_t nrows,
                                                     const int64_t* __restrict__ adj_ptr,
                                                     const int32_t* __restrict__ adj_eid,
                                                     const int32_t* __restrict__ v2, const double* __restrict__ w,
                                                     int32_t col_lo, int32_t col_hi, int32_t tile_lo,
                                                     int32_t ntiles, double scale, uint64_t seed,
                                                     double* __restrict__ Y, int64_t ldy, int tm) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t item = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; item < n * ntiles; item += nw) {
        const int64_t v = v0 + item / ntiles;
        const int32_t tile = tile_lo + (int32_t)(item - (v - v0) * ntiles);
        double acc[8];
#pragma unroll
        for (int t = 0; t < 8; t++) acc[t] = 0.0;
        for (int64_t p = adj_ptr[v]; p < adj_ptr[v + 1]; p++) {
            const int32_t e = adj_eid[p];
            const double sw = sqrt(w[e]);
            const double b = (v2[e] == (int32_t)v) ? sw : -sw;
            // lane computes call index tile*32 + lane -> u32 entries for columns 8*(tile*32+lane) .. +7
            u64x4 r = philox((uint64_t)(e - e0), (uint64_t)tile * 32 + lane, 0, 0, seed, STREAM_UNIF);
#pragma unroll
            for (int t = 0; t < 8; t++) {
                // my column j = tile*256 + lane + 32 t ; its call = j >> 3 -> source lane (lane >> 3) + 4 t
                const int src = (lane >> 3) + 4 * t;
                const uint64_t q0 = __shfl_sync(0xffffffffu, r.x, src);
                const uint64_t q1 = __shfl_sync(0xffffffffu, r.y, src);
                const uint64_t q2 = __shfl_sync(0xffffffffu, r.z, src);
                const uint64_t q3 = __shfl_sync(0xffffffffu, r.w, src);
                const int jj = lane & 7;  // (j & 7)
                const uint64_t word = (jj >> 1) == 0 ? q0 : (jj >> 1) == 1 ? q1 : (jj >> 1) == 2 ? q2 : q3;
                const uint32_t x = (jj & 1) ? (uint32_t)(word >> 32) : (uint32_t)word;
                const double u = __ddiv_rn(__dadd_rn((double)x, 0.5), 4294967296.0);
                const double h = __dsub_rn(__dmul_rn(2.0, u), 1.0);
                const double hs = __dmul_rn(h, scale);
                acc[t] = __dadd_rn(acc[t], __dmul_rn(hs, b));
            }
        }
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const int64_t col = (int64_t)tile * 256 + lane + 32 * t;
            if (col >= col_lo && col < col_hi) {
                const int64_t lc = col - col_lo;  // column of the stored block
                Y[tm ? tile_off(nrows, v, lc) : v * ldy + lc] = acc[t];
            }
        }
    }
}

void sketch_device(Context& C, const DevGraph& G, int32_t k, double scale, uint64_t seed, int uniform, double* Y,
                   int64_t ldy, int tile_major, int32_t col_lo) {
    sketch_device_part(C, G, 0, G.n, 0, k, scale, seed, uniform, Y, ldy, tile_major, col_lo);
}

// vertices [v0, v0 + nv) of G only, with edge ids counted from e0 for the signs (one graph of a union: its
// vertices and edges are contiguous, so its entries are the ones it gets alone); Y has G.n rows
void sketch_device_part(Context& C, const DevGraph& G, int64_t v0, int64_t nv, int64_t e0, int32_t k, double scale,
                        uint64_t seed, int uniform, double* Y, int64_t ldy, int tile_major, int32_t col_lo) {
    const cudaStream_t stream = C.stream;
    SSP_REQUIRE(k > 0 && (tile_major || ldy >= k), SSP_ERR_INVALID, "sketch: need 0 < k <= ld");
    SSP_REQUIRE(col_lo >= 0 && (int64_t)col_lo + k <= INT32_MAX, SSP_ERR_INVALID, "sketch: bad column range");
    const int32_t col_hi = col_lo + k;
    const int32_t tile_lo = col_lo >> 8;
    const int32_t ntiles = ((col_hi - 1) >> 8) - tile_lo + 1;
    const int64_t items = nv * ntiles;
    if (items == 0) return;
    const int threads = 256;
    const int blocks = grid_for(items * 32, threads, 148 * 16);
    if (uniform)
        k_sketch_unif<<<blocks, threads, 0, stream>>>(nv, v0, e0, G.n, G.adj_ptr, G.adj_eid, G.v2, G.w, col_lo, col_hi,
                                                        tile_lo, ntiles, scale, seed, Y, ldy, tile_major);
    else
        k_sketch_sign<<<blocks, threads, 0, stream>>>(nv, v0, e0, G.n, G.adj_ptr, G.adj_eid, G.v2, G.w, col_lo, col_hi,
                                                        tile_lo, ntiles, scale, seed, Y, ldy, tile_major);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
}

}  // namespace ssp
