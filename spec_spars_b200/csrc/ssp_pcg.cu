// ssp_pcg.cu -- a8: preconditioned conjugate gradients on all k right-hand sides at once.
//
// Reference: example_pcg_solver (custom_cg.hpp:96-274), called once per sketch column
// (example.cc:552-569).  Per column: b = rhs - mean(rhs) (:132), x0 = 0 (:140), PCG with the
// preconditioner M^{-1} r = L^{-T} D^+ L^{-1} r (:224-235, zero pivots skipped), stop once
// ||r|| <= max(abs_tol, tol ||b||) (the reference's own rule is ||r||^2 <= 2e-7, :159,213), at most
// max_iters iterations (:153), and success iff ||b - A x|| / ||b|| < 0.01 (:251-258).
//
// Layout ("tile-major", tile_off): an n x k block is stored as slabs of n x SSP_TILE values.  Every
// kernel works on one tile at a time across all rows, so the rows it gathers (one slab) stay resident
// in L2 while the sparse matrix streams.  Column reductions are two-stage with a fixed order
// (deterministic run to run) and always accumulate in FP64.
//
// Precision.  SSP_PRECISION_FP64 runs the whole iteration in FP64.  SSP_PRECISION_MIXED runs FP64
// iterative refinement around FP32 inner PCG solves: the inner SpMM, triangular solves and vector
// updates read and write FP32 (half the bytes of every gather and stream), the inner dot products
// accumulate in FP64, and after each inner solve the true residual b - A x is recomputed with the FP64
// matrix and FP64 x, so the stopping rule is checked on the same FP64 residual as in the FP64 mode.
// An inner solve stops at a fixed relative reduction (or at half the outer threshold); once a round
// fails to contract the FP64 residual by a large factor, the remaining rounds use an FP64 inner solve
// that goes straight to the outer threshold.
#include <algorithm>
#include <cmath>
#include <cstdlib>

#include <functional>

#include "ssp_internal.cuh"

namespace ssp {

constexpr int TILE = SSP_TILE;    // columns per tile
constexpr int RED_THREADS = 256;  // column reductions: (256 / TILE) row lanes x TILE columns

// mixed precision: relative reduction asked of one FP32 inner solve, and the round limit
constexpr double MIXED_INNER_REDUCTION = 1e-4;
constexpr int MIXED_MAX_ROUNDS = 40;
// a round whose FP64 residual shrinks by less than this factor (max over columns) switches the remaining
// rounds to FP64 inner solves
constexpr double MIXED_MIN_CONTRACTION = 1e-2;
// FP32 rounds after the first may take at most this many times the first round's iterations (at least
// MIXED_MIN_ROUND_ITERS); on ill-conditioned systems the FP32 recurrence stalls short of its target, and a
// round that runs into the cap hands the rest to FP64
constexpr int MIXED_ROUND_ITER_FACTOR = 2;
constexpr int MIXED_MIN_ROUND_ITERS = 20;
// the first FP32 round may take at most max_iters / MIXED_FIRST_ROUND_DIV iterations (at least
// MIXED_MIN_ROUND_ITERS): an FP32 recurrence that stalls above its target (3-D grid, n = 64^3, weights over
// six decades: still at relative residual 0.26 after 400 iterations) then leaves the rest to FP64 rounds
constexpr int MIXED_FIRST_ROUND_DIV = 4;

__host__ __device__ __forceinline__ int64_t tm_off(int64_t n, int64_t r, int64_t c) { return tile_off(n, r, c); }

// ---------------------------------------------------------------- layout conversion
__global__ void k_rm_to_tm(int64_t n, int32_t k, int64_t ldr, const double* __restrict__ src, double* __restrict__ dst,
                           int64_t ld) {
    const int64_t total = n * ld;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = i / (n * TILE), rem = i - t * n * TILE, r = rem / TILE, c = t * TILE + (rem % TILE);
        dst[i] = c < k ? src[r * ldr + c] : 0.0;
    }
}
__global__ void k_tm_to_rm(int64_t n, int32_t k, const double* __restrict__ src, double* __restrict__ dst, int64_t ldr) {
    const int64_t total = n * (int64_t)k;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / k, c = i - r * k;
        dst[r * ldr + c] = src[tm_off(n, r, c)];
    }
}

void rowmajor_to_tiles(Context& C, int64_t n, int32_t k, int64_t ldr, const double* src, double* dst) {
    const int64_t ld = ((int64_t)k + TILE - 1) / TILE * TILE;
    k_rm_to_tm<<<grid_for(n * ld, 256, 148 * 16), 256, 0, C.stream>>>(n, k, ldr, src, dst, ld);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
}
void tiles_to_rowmajor(Context& C, int64_t n, int32_t k, const double* src, double* dst, int64_t ldr) {
    k_tm_to_rm<<<grid_for(n * (int64_t)k, 256, 148 * 16), 256, 0, C.stream>>>(n, k, src, dst, ldr);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
}

// ---------------------------------------------------------------- segments (several graphs in one solve)
// A batch of graphs is solved as the disjoint union of their Laplacians: rows [row0_s, row0_{s+1}) belong to
// segment s, which owns columns [0, k_s) of the n x k block (the rest of its columns stay zero and inactive).
// Every per-column scalar (norms, thresholds, alpha, beta, activity) is per (segment, column), at index
// s * ld + c, so each graph's iterates are its own; reductions use blocks that never straddle two segments.
// A single graph is one segment with null tables, and every kernel then does exactly what it did before.
struct SegDev {
    int32_t nseg = 1;
    const int32_t* rowseg = nullptr;    // [n] segment of each row
    const int32_t* kseg = nullptr;      // [nseg] columns of each segment
    const int64_t* segrows = nullptr;   // [nseg] rows of each segment
    const int64_t* blk_row = nullptr;   // [nparts + 1] row boundaries of the reduction blocks
    const int32_t* blk_seg = nullptr;   // [nparts] segment of each reduction block
    const int32_t* part_start = nullptr;  // [nseg + 1] first reduction block of each segment
};
__device__ __forceinline__ int64_t seg_of_row(const SegDev& G, int64_t row) { return G.rowseg ? G.rowseg[row] : 0; }
// rows of reduction block blockIdx.x and the state offset (segment * ld) of its segment
__device__ __forceinline__ void red_block(const SegDev& G, int64_t n, int64_t rows_per_blk, int64_t ld, int64_t& r0,
                                          int64_t& r1, int64_t& sbase) {
    if (G.blk_row) {
        r0 = G.blk_row[blockIdx.x];
        r1 = G.blk_row[blockIdx.x + 1];
        sbase = (int64_t)G.blk_seg[blockIdx.x] * ld;
    } else {
        r0 = (int64_t)blockIdx.x * rows_per_blk;
        r1 = min(n, r0 + rows_per_blk);
        sbase = 0;
    }
}

// Rows of converged graphs (several graphs at once): act[s * ntiles + t] says whether graph s still has an
// active column in tile t; the SpMM and the triangular solves skip the rows of inactive (graph, tile) pairs,
// whose values no active column reads (alpha is 0 there).  A null act (one graph) skips nothing.
struct RowAct {
    const int32_t* act = nullptr;
    const int32_t* rowseg = nullptr;  // graph of each vertex
    int32_t ntiles = 0;
};
__device__ __forceinline__ bool row_on(const RowAct& A, int64_t vertex, int64_t tile) {
    return !A.act || A.act[(int64_t)A.rowseg[vertex] * A.ntiles + tile];
}
__global__ void k_seg_tile_active(int32_t nseg, int32_t ntiles, int64_t ld, const int32_t* __restrict__ active,
                                  int32_t* __restrict__ act) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)nseg * ntiles;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t sg = i / ntiles, t = i - sg * ntiles;
        int32_t a = 0;
        for (int c = 0; c < TILE; c++) a |= active[sg * ld + t * TILE + c];
        act[i] = a;
    }
}

// ---------------------------------------------------------------- column reductions
enum ColOp { OP_SUM = 0, OP_DOT = 1, OP_SQ = 2, OP_SQDIFF_CENTERED = 3 };

// grid (nparts, ntiles); thread = (row lane = tid / 8, column = tid % 8); part[blk][col]
template <int OP, class T>
__global__ void __launch_bounds__(RED_THREADS) k_colred_partial(int64_t n, const T* __restrict__ a,
                                                                const T* __restrict__ b,
                                                                const double* __restrict__ mean, int64_t rows_per_blk,
                                                                int64_t ld, double* __restrict__ part, SegDev G) {
    __shared__ double s[RED_THREADS];
    const int64_t t = blockIdx.y;
    const int c = threadIdx.x % TILE, rl = threadIdx.x / TILE;
    int64_t r0, r1, sb;
    red_block(G, n, rows_per_blk, ld, r0, r1, sb);
    const T* at = a + t * n * TILE;
    const T* bt = b ? b + t * n * TILE : nullptr;
    const double mu = (OP == OP_SQDIFF_CENTERED) ? mean[sb + t * TILE + c] : 0.0;
    double acc = 0.0;
    for (int64_t r = r0 + rl; r < r1; r += RED_THREADS / TILE) {
        const double x = (double)at[r * TILE + c];
        if (OP == OP_SUM) acc += x;
        else if (OP == OP_DOT) acc += x * (double)bt[r * TILE + c];
        else if (OP == OP_SQ) acc += x * x;
        else {
            const double d = (x - mu) - (double)bt[r * TILE + c];  // (Y - mean) - A x
            acc += d * d;
        }
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x < TILE) {
        double tt = s[threadIdx.x];
        for (int i = 1; i < RED_THREADS / TILE; i++) tt += s[i * TILE + threadIdx.x];
        part[(int64_t)blockIdx.x * ld + t * TILE + threadIdx.x] = tt;
    }
}

// out[c] = sum over parts of part[i][c]: a block per 32 columns, warp w sums the parts i = w (mod FIN_WARPS) two
// at a time, then the warps' sums are added in warp order (fixed order: deterministic).  Hundreds of parts per
// column (the SpMM's p.q partials) are then 16-way parallel instead of one thread's dependent chain.
constexpr int FIN_WARPS = 16;
// With segments, out[s * ld + c] sums the parts of segment s's blocks, in the same order.
__global__ void __launch_bounds__(FIN_WARPS * 32) k_colred_final(int64_t ld, int nparts, const double* __restrict__ part,
                                                                  double* __restrict__ out, SegDev G) {
    __shared__ double s[FIN_WARPS][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t o = (int64_t)blockIdx.x * 32 + lane;
    const int64_t seg = o / ld, c = o - seg * ld;
    const bool in = o < (int64_t)G.nseg * ld;
    const int p0 = G.part_start && in ? G.part_start[seg] : 0;
    const int np = G.part_start && in ? G.part_start[seg + 1] - p0 : nparts;
    double a0 = 0.0, a1 = 0.0;
    if (in) {
        int i = w;
        for (; i + FIN_WARPS < np; i += 2 * FIN_WARPS) {
            a0 += part[(int64_t)(p0 + i) * ld + c];
            a1 += part[(int64_t)(p0 + i + FIN_WARPS) * ld + c];
        }
        if (i < np) a0 += part[(int64_t)(p0 + i) * ld + c];
    }
    s[w][lane] = a0 + a1;
    __syncthreads();
    if (w == 0 && in) {
        double t = 0.0;
        for (int j = 0; j < FIN_WARPS; j++) t += s[j][lane];
        out[o] = t;
    }
}
static void colred_final(Context& C, int64_t ld, int nparts, const double* part, double* out,
                         const SegDev& G = SegDev()) {
    k_colred_final<<<(unsigned)ceil_div<int64_t>((int64_t)G.nseg * ld, 32), FIN_WARPS * 32, 0, C.stream>>>(
        ld, nparts, part, out, G);
}

struct Reducer {
    Context* C;
    int64_t n, ld;
    int nparts;
    int64_t rows_per_blk;
    double* part;
    SegDev G;  // segment tables (the block tables are filled in by init when there are several segments)
    // row0: nseg + 1 segment row starts on the host (empty: one segment); G's rowseg/kseg/segrows are the
    // caller's
    void init(Context& c, int64_t n_, int64_t ld_, const char* tag = "pcg_red_part", const SegDev& segs = SegDev(),
              const std::vector<int64_t>* row0 = nullptr) {
        C = &c;
        n = n_;
        ld = ld_;
        G = segs;
        const int64_t ntiles = ld / TILE;
        int64_t target = std::max<int64_t>(8, std::min<int64_t>(1184 / std::max<int64_t>(1, ntiles) + 1, 1024));
        rows_per_blk = std::max<int64_t>(RED_THREADS / TILE, ceil_div<int64_t>(n, target));
        if (G.nseg <= 1 || !row0) {
            nparts = (int)ceil_div<int64_t>(n, rows_per_blk);
        } else {
            // blocks of at most rows_per_blk rows inside each segment
            std::vector<int64_t> brow;
            std::vector<int32_t> bseg, pstart;
            for (int32_t sg = 0; sg < G.nseg; sg++) {
                pstart.push_back((int32_t)bseg.size());
                for (int64_t r = (*row0)[sg]; r < (*row0)[sg + 1]; r += rows_per_blk) {
                    brow.push_back(r);
                    bseg.push_back(sg);
                }
            }
            pstart.push_back((int32_t)bseg.size());
            brow.push_back(n);
            nparts = (int)bseg.size();
            int64_t* d_brow = c.ws.get_t<int64_t>(std::string(tag) + "_brow", brow.size());
            int32_t* d_bseg = c.ws.get_t<int32_t>(std::string(tag) + "_bseg", bseg.size() + 1);
            int32_t* d_pst = c.ws.get_t<int32_t>(std::string(tag) + "_pstart", pstart.size());
            SSP_CUDA(cudaMemcpyAsync(d_brow, brow.data(), sizeof(int64_t) * brow.size(), cudaMemcpyHostToDevice,
                                     c.stream));
            SSP_CUDA(cudaMemcpyAsync(d_bseg, bseg.data(), sizeof(int32_t) * bseg.size(), cudaMemcpyHostToDevice,
                                     c.stream));
            SSP_CUDA(cudaMemcpyAsync(d_pst, pstart.data(), sizeof(int32_t) * pstart.size(), cudaMemcpyHostToDevice,
                                     c.stream));
            SSP_CUDA(cudaStreamSynchronize(c.stream));
            G.blk_row = d_brow;
            G.blk_seg = d_bseg;
            G.part_start = d_pst;
        }
        part = c.ws.get_t<double>(tag, (size_t)nparts * ld);
    }
    template <int OP, class T>
    void run(const T* a, const T* b, double* out, const double* mean = nullptr) {
        dim3 grid((unsigned)nparts, (unsigned)(ld / TILE));
        k_colred_partial<OP, T><<<grid, RED_THREADS, 0, C->stream>>>(n, a, b, mean, rows_per_blk, ld, part, G);
        colred_final(*C, ld, nparts, part, out, G);
        SSP_CHECK_LAUNCH();
        C->kernels_launched += 2;
    }
    void finish(double* out) {
        colred_final(*C, ld, nparts, part, out, G);
        SSP_CHECK_LAUNCH();
        C->kernels_launched++;
    }
};

// ---------------------------------------------------------------- elementwise (grid.y = tile)
// r = Y - mean(Y) over each segment's rows for its columns (0 elsewhere), x = 0, mean per (segment, column)
__global__ void k_center(int64_t n, int32_t k, int64_t ld, const double* __restrict__ Y,
                         const double* __restrict__ colsum, double* __restrict__ r, double* __restrict__ x,
                         double* __restrict__ mean, SegDev G) {
    const int64_t t = blockIdx.y;
    const int64_t cnt = n * TILE;
    if (blockIdx.x == 0 && threadIdx.x < TILE)
        for (int32_t sg = 0; sg < G.nseg; sg++) {
            const int64_t c = t * TILE + threadIdx.x;
            const int32_t kk = G.kseg ? G.kseg[sg] : k;
            const int64_t nr = G.segrows ? G.segrows[sg] : n;
            mean[sg * ld + c] = c < kk ? colsum[sg * ld + c] / (double)nr : 0.0;
        }
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = t * TILE + (i % TILE);
        const int64_t o = t * cnt + i;
        const int64_t sg = seg_of_row(G, i / TILE);
        const int32_t kk = G.kseg ? G.kseg[sg] : k;
        const int64_t nr = G.segrows ? G.segrows[sg] : n;
        const double mu = c < kk ? colsum[sg * ld + c] / (double)nr : 0.0;
        r[o] = c < kk ? Y[o] - mu : 0.0;
        x[o] = 0.0;
    }
}

// r -= alpha q ; partial ||r||^2 per column (FP64 accumulation).  The matching x += alpha p is deferred to
// the next p update (k_update_xp), which reads p anyway, or to k_axpy_x after the last iteration: x gets
// the same additions in the same order, one n x k stream fewer per iteration.
template <class T>
__global__ void __launch_bounds__(RED_THREADS) k_axpy_r_rr(int64_t n, const double* __restrict__ alpha,
                                                           const T* __restrict__ q, T* __restrict__ r,
                                                           int64_t rows_per_blk, int64_t ld, double* __restrict__ part,
                                                           SegDev G) {
    __shared__ double s[RED_THREADS];
    const int64_t t = blockIdx.y;
    const int c = threadIdx.x % TILE, rl = threadIdx.x / TILE;
    int64_t r0, r1, sb;
    red_block(G, n, rows_per_blk, ld, r0, r1, sb);
    const double a64 = alpha[sb + t * TILE + c];
    const T a = (T)a64;
    const int64_t base = t * n * TILE;
    double acc = 0.0;
    for (int64_t row = r0 + rl; row < r1; row += RED_THREADS / TILE) {
        const int64_t o = base + row * TILE + c;
        T rv = r[o];
        if (a64 != 0.0) {
            rv -= a * q[o];
            r[o] = rv;
        }
        acc += (double)rv * (double)rv;
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x < TILE) {
        double tt = s[threadIdx.x];
        for (int i = 1; i < RED_THREADS / TILE; i++) tt += s[i * TILE + threadIdx.x];
        part[(int64_t)blockIdx.x * ld + t * TILE + threadIdx.x] = tt;
    }
}

// x += alpha p (the previous step's alpha and p), then p = z + beta p
template <class T>
__global__ void k_update_xp(int64_t n, int64_t ld, const double* __restrict__ alpha, const double* __restrict__ beta,
                            const T* __restrict__ z, T* __restrict__ p, T* __restrict__ x, SegDev G) {
    const int64_t t = blockIdx.y;
    const int64_t cnt = n * TILE;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = t * cnt + i;
        const int64_t c = seg_of_row(G, i / TILE) * ld + t * TILE + (i % TILE);
        const double a64 = alpha[c];
        const T pv = p[o];
        if (a64 != 0.0) x[o] += (T)a64 * pv;
        p[o] = z[o] + (T)beta[c] * pv;
    }
}

// the last step's x += alpha p
template <class T>
__global__ void k_axpy_x(int64_t n, int64_t ld, const double* __restrict__ alpha, const T* __restrict__ p,
                         T* __restrict__ x, SegDev G) {
    const int64_t t = blockIdx.y;
    const int64_t cnt = n * TILE;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = t * cnt + i;
        const double a64 = alpha[seg_of_row(G, i / TILE) * ld + t * TILE + (i % TILE)];
        if (a64 != 0.0) x[o] += (T)a64 * p[o];
    }
}

// ---------------------------------------------------------------- mixed-precision helpers
__global__ void k_d2f(int64_t count, const double* __restrict__ src, float* __restrict__ dst) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}
__global__ void k_f2d(int64_t count, const float* __restrict__ src, double* __restrict__ dst) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

// inner right-hand side: the FP64 residual of the columns still active, rounded to T; zero elsewhere
// (runs in place when T is double)
template <class T>
__global__ void k_rhs_masked(int64_t n, int64_t ld, const double* r64, const int32_t* __restrict__ active, T* rin,
                             SegDev G) {
    const int64_t t = blockIdx.y;
    const int64_t cnt = n * TILE;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = t * cnt + i;
        rin[o] = active[seg_of_row(G, i / TILE) * ld + t * TILE + (i % TILE)] ? (T)r64[o] : (T)0;
    }
}

template <class T>
__global__ void k_add_into(int64_t count, const T* __restrict__ e, double* __restrict__ x) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        x[i] += (double)e[i];
}

// r = (Y - mean) - q with partial ||r||^2 per column: the true FP64 residual after a refinement round
__global__ void __launch_bounds__(RED_THREADS) k_true_resid(int64_t n, int32_t k, const double* __restrict__ Y,
                                                            const double* __restrict__ mean,
                                                            const double* __restrict__ q, double* __restrict__ r,
                                                            int64_t rows_per_blk, int64_t ld, double* __restrict__ part,
                                                            SegDev G) {
    __shared__ double s[RED_THREADS];
    const int64_t t = blockIdx.y;
    const int c = threadIdx.x % TILE, rl = threadIdx.x / TILE;
    int64_t r0, r1, sb;
    red_block(G, n, rows_per_blk, ld, r0, r1, sb);
    const int64_t col = t * TILE + c;
    if (G.kseg) k = G.kseg[sb / ld];
    const double mu = mean[sb + col];
    const int64_t base = t * n * TILE;
    double acc = 0.0;
    for (int64_t row = r0 + rl; row < r1; row += RED_THREADS / TILE) {
        const int64_t o = base + row * TILE + c;
        const double rv = col < k ? (Y[o] - mu) - q[o] : 0.0;
        r[o] = rv;
        acc += rv * rv;
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x < TILE) {
        double tt = s[threadIdx.x];
        for (int i = 1; i < RED_THREADS / TILE; i++) tt += s[i * TILE + threadIdx.x];
        part[(int64_t)blockIdx.x * ld + t * TILE + threadIdx.x] = tt;
    }
}

// ---------------------------------------------------------------- per-column scalars
struct ColState {
    double* bnorm2;
    double* thr;
    double* rz;
    double* rz_new;
    double* pq;
    double* rr;
    double* alpha;
    double* beta;
    int32_t* active;
    int32_t* iters;
    int64_t* nactive;
};

static ColState make_colstate(Context& C, int64_t ld, const std::string& tag) {
    double* v = C.ws.get_t<double>(tag + "_cols", 8 * ld);
    int32_t* iv = C.ws.get_t<int32_t>(tag + "_coli", 2 * ld);
    int64_t* na = C.ws.get_t<int64_t>(tag + "_nactive", 1);
    return ColState{v, v + ld, v + 2 * ld, v + 3 * ld, v + 4 * ld, v + 5 * ld, v + 6 * ld, v + 7 * ld, iv, iv + ld, na};
}

// state entries c = segment * ld + column; a column past its segment's k_s is inactive
__global__ void k_cols_init(int64_t ld, int32_t k, double tol, double abs_tol, ColState S, SegDev G) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < (int64_t)G.nseg * ld;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int32_t kk = G.kseg ? G.kseg[c / ld] : k;
        double bn = sqrt(S.bnorm2[c]);
        double thr = tol * bn;
        if (abs_tol > thr) thr = abs_tol;
        S.thr[c] = thr;
        S.rr[c] = S.bnorm2[c];
        int act = (c % ld < kk) && (bn > thr);
        S.active[c] = act;
        S.iters[c] = 0;
        S.alpha[c] = 0.0;
        S.beta[c] = 0.0;
        if (act) atomicAdd((unsigned long long*)S.nactive, 1ull);
    }
}

// inner solve of a refinement round: stop at a relative reduction `reduction` of its right-hand side, or
// once below half the outer threshold of the column (no point solving past what the outer test needs)
__global__ void k_cols_init_inner(int64_t ld, int32_t k, double reduction, const double* __restrict__ thr_out,
                                  ColState S, SegDev G) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < (int64_t)G.nseg * ld;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int32_t kk = G.kseg ? G.kseg[c / ld] : k;
        const double bn = sqrt(S.bnorm2[c]);
        double thr = reduction * bn;
        const double half_out = 0.5 * thr_out[c];
        if (half_out > thr) thr = half_out;
        S.thr[c] = thr;
        S.rr[c] = S.bnorm2[c];
        const int act = (c % ld < kk) && (bn > thr);
        S.active[c] = act;
        S.iters[c] = 0;
        S.alpha[c] = 0.0;
        S.beta[c] = 0.0;
        if (act) atomicAdd((unsigned long long*)S.nactive, 1ull);
    }
}

__global__ void k_cols_alpha(int64_t cnt, ColState S) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < cnt; c += (int64_t)gridDim.x * blockDim.x)
        S.alpha[c] = S.active[c] ? S.rz[c] / S.pq[c] : 0.0;
}

__global__ void k_cols_check(int64_t cnt, int32_t it, ColState S) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < cnt; c += (int64_t)gridDim.x * blockDim.x) {
        if (!S.active[c]) continue;
        S.iters[c] = it;
        if (sqrt(S.rr[c]) <= S.thr[c]) S.active[c] = 0;
        else atomicAdd((unsigned long long*)S.nactive, 1ull);
    }
}

__global__ void k_cols_beta(int64_t cnt, ColState S) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < cnt; c += (int64_t)gridDim.x * blockDim.x) {
        double b = 0.0;
        if (S.active[c]) b = S.rz_new[c] / S.rz[c];
        S.beta[c] = b;
        S.rz[c] = S.rz_new[c];
    }
}

// outer test of a refinement round on the true residual: adds the round's inner iterations to the
// column's count, deactivates converged columns, and records the largest residual ratio new/old
__global__ void k_cols_outer(int64_t cnt, const int32_t* __restrict__ inner_iters, const double* __restrict__ rr_new,
                             ColState S, double* __restrict__ worst_ratio) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < cnt; c += (int64_t)gridDim.x * blockDim.x) {
        if (!S.active[c]) continue;
        S.iters[c] += inner_iters[c];
        const double before = S.rr[c], after = rr_new[c];
        S.rr[c] = after;
        if (sqrt(after) <= S.thr[c]) {
            S.active[c] = 0;
        } else {
            atomicAdd((unsigned long long*)S.nactive, 1ull);
            const double ratio = before > 0 ? sqrt(after / before) : 1.0;
            // ratios are non-negative: their IEEE bit patterns order like the values
            atomicMax((unsigned long long*)worst_ratio, (unsigned long long)__double_as_longlong(ratio));
        }
    }
}

// ---------------------------------------------------------------- the iteration loop on the device
// The PCG iterations after the first run as the body of a CUDA-graph WHILE node: the body advances the
// iteration counter on the device, runs the convergence check, and k_loop_ctl keeps the loop going only while
// some column is active and fewer than max_iters iterations have run, so the loop ends by itself without a
// host round trip per iteration.
__global__ void k_it_set(int32_t* it, int32_t v) { *it = v; }
__global__ void k_it_next(int32_t* it) { *it += 1; }

__global__ void k_cols_check_at(int64_t cnt, const int32_t* __restrict__ it, ColState S) {
    const int32_t i = *it;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < cnt; c += (int64_t)gridDim.x * blockDim.x) {
        if (!S.active[c]) continue;
        S.iters[c] = i;
        if (sqrt(S.rr[c]) <= S.thr[c]) S.active[c] = 0;
        else atomicAdd((unsigned long long*)S.nactive, 1ull);
    }
}

__global__ void k_loop_ctl(cudaGraphConditionalHandle h, const int64_t* __restrict__ nactive,
                           const int32_t* __restrict__ it, int32_t max_iters) {
    cudaGraphSetConditional(h, (*nactive > 0 && *it < max_iters) ? 1u : 0u);
}

struct LoopGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~LoopGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

// ---------------------------------------------------------------- SpMM and triangular solves
// Warp per row; lane = slot * W + column, W = the columns handled (TILE, or 8 when at most 8 are real).
// ---------------------------------------------------------------- chunked gather (SpMM-shaped work)
// A chunk is a run of consecutive stored rows with at most CHUNK_CAP entries and CHUNK_ROWS rows (or
// one longer row).  Each warp owns whole chunks: it stages the chunk's (index, value) pairs in its own
// shared-memory slice with coalesced streaming loads (the matrix is read once per tile and should not
// evict the gathered slab from L2), then every (row, column) lane pair sums its row with independent
// gathers from the tile slab.  Warps never wait for each other.  Modes: SpMM (+ p.q partials), SpMM
// adding into its output (the second and later column slabs of the matrix), forward solve, backward solve.
enum { M_SPMM = 0, M_FWD = 1, M_BWD = 2, M_SPMM_ACC = 3, M_FWD_LAST = 4 };
constexpr int CH_THREADS = 256;
// independent gathers in flight per lane in the chunk kernels (powers of two).  Measured on B200 at ER n = 1M,
// k = 1327: 8 for the SpMM takes it from 48 to 38 ms; the level solves are faster with 4 (19 against 22 ms).
#ifndef SSP_GATHER_UNROLL_SPMM
#define SSP_GATHER_UNROLL_SPMM 8
#endif
#ifndef SSP_GATHER_UNROLL_SOLVE
#define SSP_GATHER_UNROLL_SOLVE 4
#endif
constexpr int CH_WARPS = CH_THREADS / 32;
constexpr int MINB_SPMM = 6, MINB_FWD = 6, MINB_BWD = 5;

template <int MODE, class T>
__device__ __forceinline__ void chunk_epilogue(T* out, const T* aux, const T* xt, int64_t toff, int64_t v, int col,
                                               T acc, double& dot, bool want_dot, const T* dlast) {
    const int64_t o = toff + v * TILE + col;
    if (MODE == M_SPMM || MODE == M_SPMM_ACC) {
        // q streams out (evict-first), so it does not push the gathered slab out of L2
        if (MODE == M_SPMM_ACC) acc += __ldcs(out + o);
        __stcs(out + o, acc);
        if (want_dot) dot += (double)acc * (double)xt[v * TILE + col];
    } else if (MODE == M_FWD) {
        out[o] = aux[o] - acc;
    } else if (MODE == M_FWD_LAST) {
        // the forward value, then the backward solve's step for a row with an empty column
        const T yu = aux[o] - acc;
        const T d = dlast[v];
        out[o] = (d != (T)0 ? yu / d : yu) - (T)0;
    } else {
        const T d = aux[v];
        const T yu = out[o];
        out[o] = (d != (T)0 ? yu / d : yu) - acc;
    }
}

// Grid: x over chunks, y over (tile, sub-tile): a tile's TILE columns are covered by nsub = TILE / W warps'
// column ranges (nsub = 1 for the full-width layout, or for the narrow one when only W columns are real).
// MINB: resident blocks per SM asked of the compiler.  The SpMM asks for six (its registers would otherwise
// allow five: FP32 SpMM 29.7 -> 22.6 ms at ER n = 1M); the level solves ask for what their own register
// choice gives (forward 6, backward 5; forcing six on the backward solve cost the preconditioner 7 %).
// Keeping the body in the kernel itself matters: moved into a __device__ function holding the shared
// arrays, the FP32 SpMM took 39 ms instead of 22.6 (twice the long-scoreboard stalls per issue).
template <int MODE, class T, int W, int MINB>
__global__ void __launch_bounds__(CH_THREADS, MINB)
    k_chunked(int64_t n, const int32_t* __restrict__ cstart, int32_t nchunks, const int64_t* __restrict__ ptr,
              const int32_t* __restrict__ idx, const T* __restrict__ val, const int32_t* __restrict__ rowmap,
              const T* xsrc, T* out, const T* __restrict__ aux, int64_t ld, double* __restrict__ part,
              int32_t kcols, int nsub, const T* __restrict__ dlast = nullptr, RowAct ra = RowAct()) {
    __shared__ int32_t s_idx[CH_WARPS][CHUNK_CAP];
    __shared__ T s_val[CH_WARPS][CHUNK_CAP];
    __shared__ int32_t s_ptr[CH_WARPS][CHUNK_ROWS + 1];
    __shared__ int32_t s_row[CH_WARPS][CHUNK_ROWS];
    __shared__ double s_red[CH_THREADS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t t = blockIdx.y / nsub;
    const int c0 = (int)(blockIdx.y % nsub) * W;  // first column of this block's sub-tile
    const int64_t toff = t * n * TILE;
    const T* xt = xsrc + toff;
    int32_t* si = s_idx[w];
    T* sv = s_val[w];
    int32_t* sp = s_ptr[w];
    int32_t* sr = s_row[w];
    constexpr int SLOTS_W = 32 / W;
    constexpr bool SPMM = MODE == M_SPMM || MODE == M_SPMM_ACC;
    const bool want_dot = SPMM && part != nullptr;
    double dot = 0.0;  // SpMM: per-lane partial of p.q for column (lane % W)
    for (int32_t c = blockIdx.x * CH_WARPS + w; c < nchunks; c += gridDim.x * CH_WARPS) {
        const int32_t r0 = cstart[c], r1 = cstart[c + 1];
        const int64_t e0 = ptr[r0], e1 = ptr[r1];
        const int64_t ne = e1 - e0;
        if (ne <= CHUNK_CAP) {
            for (int64_t i = lane; i < ne; i += 32) {
                si[i] = __ldcs(idx + e0 + i);
                sv[i] = __ldcs(val + e0 + i);
            }
            // the chunk's row pointers and vertex ids (level solves: storage row -> vertex) staged together
            for (int32_t i = lane; i <= r1 - r0; i += 32) {
                sp[i] = (int32_t)(ptr[r0 + i] - e0);
                if (i < r1 - r0) sr[i] = rowmap ? rowmap[r0 + i] : r0 + i;
            }
            __syncwarp();
            const int32_t pairs = (r1 - r0) * W;
            for (int32_t pr = lane; pr < pairs; pr += 32) {
                const int32_t rr = pr / W, col = c0 + pr % W;
                const int64_t vrow = sr[rr];
                const bool on = row_on(ra, vrow, t);
                const bool live = on && t * TILE + col < kcols;
                const int32_t q0 = sp[rr], q1 = live ? sp[rr + 1] : q0;
                // GATHER_UNROLL independent accumulators, summed as a pairwise tree
                constexpr int GATHER_UNROLL = SPMM ? SSP_GATHER_UNROLL_SPMM : SSP_GATHER_UNROLL_SOLVE;
                T a[GATHER_UNROLL];
#pragma unroll
                for (int u = 0; u < GATHER_UNROLL; u++) a[u] = 0;
                int32_t q = q0;
                for (; q + GATHER_UNROLL - 1 < q1; q += GATHER_UNROLL) {
#pragma unroll
                    for (int u = 0; u < GATHER_UNROLL; u++) a[u] += sv[q + u] * xt[(int64_t)si[q + u] * TILE + col];
                }
                if (GATHER_UNROLL > 4 && q + 3 < q1) {  // short rows (a slab's share of a row) still get 4 in flight
#pragma unroll
                    for (int u = 0; u < 4; u++) a[u] += sv[q + u] * xt[(int64_t)si[q + u] * TILE + col];
                    q += 4;
                }
                for (; q < q1; q++) a[0] += sv[q] * xt[(int64_t)si[q] * TILE + col];
#pragma unroll
                for (int h = 1; h < GATHER_UNROLL; h <<= 1)
#pragma unroll
                    for (int u = 0; u < GATHER_UNROLL; u += 2 * h) a[u] += a[u + h];
                if (on) chunk_epilogue<MODE, T>(out, aux, xt, toff, vrow, col, a[0], dot, want_dot, dlast);
            }
            __syncwarp();
        } else {
            // One long row: (32 / W) entry slots x W columns per step.  The sum does not depend on W: entry i
            // of the row goes to virtual accumulator i mod LONG_ACC (each summed in entry order), and the
            // accumulators are combined by a fixed tree, highest index bit first.  A lane of slot s holds the
            // accumulators s + SLOTS_W j; it combines their high bits itself, the slot bits are combined
            // across lanes afterwards (offset 16 first), so a level solved with any column width W gives
            // the same values bit for bit -- which lets the launch shapes be chosen by measurement.
            constexpr int LONG_ACC = 4, NA = LONG_ACC / SLOTS_W;
            static_assert(NA >= 1 && LONG_ACC % SLOTS_W == 0, "column width below 8");
            const int slot = lane / W, col = c0 + lane % W;
            const int64_t vr0 = rowmap ? rowmap[r0] : r0;
            const bool on = row_on(ra, vr0, t);
            const int64_t qe = on && t * TILE + col < kcols ? e1 : e0;
            T a[NA];
#pragma unroll
            for (int j = 0; j < NA; j++) a[j] = 0;
            int64_t q = e0 + slot;
            for (; q + (NA - 1) * SLOTS_W < qe; q += NA * SLOTS_W) {
#pragma unroll
                for (int j = 0; j < NA; j++)
                    a[j] += __ldcs(val + q + j * SLOTS_W) * xt[(int64_t)__ldcs(idx + q + j * SLOTS_W) * TILE + col];
            }
#pragma unroll
            for (int j = 0; j < NA - 1; j++)
                if (q + j * SLOTS_W < qe)
                    a[j] += __ldcs(val + q + j * SLOTS_W) * xt[(int64_t)__ldcs(idx + q + j * SLOTS_W) * TILE + col];
#pragma unroll
            for (int h = NA / 2; h >= 1; h >>= 1)
#pragma unroll
                for (int j = 0; j < h; j++) a[j] += a[j + h];
            T acc = a[0];
#pragma unroll
            for (int o = 16; o >= W; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane < W && on) chunk_epilogue<MODE, T>(out, aux, xt, toff, vr0, col, acc, dot, want_dot, dlast);
        }
    }
    if (want_dot) {
        s_red[threadIdx.x] = dot;
        __syncthreads();
        if (threadIdx.x < TILE) {
            double tt = 0.0;
            if (threadIdx.x < W)
                for (int i = 0; i < CH_THREADS / W; i++) tt += s_red[i * W + threadIdx.x];
            part[(int64_t)blockIdx.x * ld + t * TILE + threadIdx.x] = tt;
        }
    }
}

// The final product of a solve, one tile per launch, also forming the squared diff norms of the edges from
// the rows it gathers: the edge of an entry with row < column (eid >= 0) gets, per tile, the xor-butterfly
// sum over the tile's 32 columns of (x[row] - x[col])^2 (0 for columns past k), added to d2 in tile order
// (first: stored) -- diff_norms_device's order.  All 32 lanes of a warp walk the same row and entry, so the
// eid test and the butterfly are warp-uniform.  q with four accumulators (eight gathers in flight with
// interleaved butterflies need 64 registers and ran slower: 1260 against 1231 ms per ER 1M step).
__global__ void __launch_bounds__(CH_THREADS) k_spmm_diff(int64_t n, const int32_t* __restrict__ cstart,
                                                          int32_t nchunks, const int64_t* __restrict__ ptr,
                                                          const int32_t* __restrict__ idx,
                                                          const double* __restrict__ val,
                                                          const int32_t* __restrict__ eid, const double* xt,
                                                          double* qt, int32_t kcols, double* __restrict__ d2,
                                                          int first) {
    __shared__ int32_t s_idx[CH_WARPS][CHUNK_CAP];
    __shared__ double s_val[CH_WARPS][CHUNK_CAP];
    __shared__ int32_t s_eid[CH_WARPS][CHUNK_CAP];
    __shared__ int32_t s_ptr[CH_WARPS][CHUNK_ROWS + 1];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const bool live = lane < kcols;
    int32_t* si = s_idx[w];
    double* sv = s_val[w];
    int32_t* se = s_eid[w];
    int32_t* sp = s_ptr[w];
    // one entry: its gathered value g, and the squared difference into d2 when the entry names an edge
    auto edge = [&](int32_t e, double xo, double g) {
        if (e < 0) return;  // warp-uniform
        const double dx = live ? __dsub_rn(xo, g) : 0.0;
        double sq = __dmul_rn(dx, dx);
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) sq = __dadd_rn(sq, __shfl_xor_sync(0xffffffffu, sq, o));
        if (lane == 0) d2[e] = first ? sq : __dadd_rn(d2[e], sq);
    };
    for (int32_t c = blockIdx.x * CH_WARPS + w; c < nchunks; c += gridDim.x * CH_WARPS) {
        const int32_t r0 = cstart[c], r1 = cstart[c + 1];
        const int64_t e0 = ptr[r0], e1 = ptr[r1];
        const int64_t ne = e1 - e0;
        if (ne <= CHUNK_CAP) {
            for (int64_t i = lane; i < ne; i += 32) {
                si[i] = __ldcs(idx + e0 + i);
                sv[i] = __ldcs(val + e0 + i);
                se[i] = __ldcs(eid + e0 + i);
            }
            for (int32_t i = lane; i <= r1 - r0; i += 32) sp[i] = (int32_t)(ptr[r0 + i] - e0);
            __syncwarp();
            for (int32_t rr = 0; rr < r1 - r0; rr++) {
                const int64_t row = r0 + rr;
                const double xo = live ? xt[row * TILE + lane] : 0.0;
                const int32_t q0 = sp[rr], q1 = sp[rr + 1];
                double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
                int32_t q = q0;
                for (; q + 3 < q1; q += 4) {
                    const double g0 = live ? xt[(int64_t)si[q] * TILE + lane] : 0.0;
                    const double g1 = live ? xt[(int64_t)si[q + 1] * TILE + lane] : 0.0;
                    const double g2 = live ? xt[(int64_t)si[q + 2] * TILE + lane] : 0.0;
                    const double g3 = live ? xt[(int64_t)si[q + 3] * TILE + lane] : 0.0;
                    a0 += sv[q] * g0;
                    a1 += sv[q + 1] * g1;
                    a2 += sv[q + 2] * g2;
                    a3 += sv[q + 3] * g3;
                    edge(se[q], xo, g0);
                    edge(se[q + 1], xo, g1);
                    edge(se[q + 2], xo, g2);
                    edge(se[q + 3], xo, g3);
                }
                for (; q < q1; q++) {
                    const double g = live ? xt[(int64_t)si[q] * TILE + lane] : 0.0;
                    a0 += sv[q] * g;
                    edge(se[q], xo, g);
                }
                __stcs(qt + row * TILE + lane, (a0 + a1) + (a2 + a3));
            }
            __syncwarp();
        } else {
            // one long row, lane = column
            const double xo = live ? xt[(int64_t)r0 * TILE + lane] : 0.0;
            double a0 = 0, a1 = 0;
            int64_t q = e0;
            for (; q + 1 < e1; q += 2) {
                const int32_t i0 = __ldcs(idx + q), i1 = __ldcs(idx + q + 1);
                const double g0 = live ? xt[(int64_t)i0 * TILE + lane] : 0.0;
                const double g1 = live ? xt[(int64_t)i1 * TILE + lane] : 0.0;
                a0 += __ldcs(val + q) * g0;
                a1 += __ldcs(val + q + 1) * g1;
                edge(__ldcs(eid + q), xo, g0);
                edge(__ldcs(eid + q + 1), xo, g1);
            }
            if (q < e1) {
                const double g = live ? xt[(int64_t)__ldcs(idx + q) * TILE + lane] : 0.0;
                a0 += __ldcs(val + q) * g;
                edge(__ldcs(eid + q), xo, g);
            }
            __stcs(qt + (int64_t)r0 * TILE + lane, a0 + a1);
        }
    }
}

// blocks per tile: about one wave of resident blocks, so the gathered slab of the tile being worked
// on is the only one live in L2
static int chunk_blocks(int32_t nchunks) {
    return std::max(1, std::min((nchunks + CH_WARPS - 1) / CH_WARPS, 148 * 6));
}

// Runs of thin levels: the k columns are independent, so one block per column tile walks the run's steps
// (rows grouped by dependency depth, DevFactor::SolveRun) on its own, with only block barriers between
// steps (its own writes are the only values it reads back).  y is read and written in place: no read-only
// cache path.  A step with fewer rows than warps splits each row's entries over several warps (partial sums
// added in warp order), so a lone row costs about one gather latency instead of one per entry.
constexpr int RUN_THREADS = 512;
constexpr int RUN_WARPS = RUN_THREADS / 32;

// one warp's share of a row: entries ptr[row] + sub * SLOTS_W + slot, stepping g * SLOTS_W, four in flight,
// summed over the slots; every lane returns its column's partial
template <class T, int W>
__device__ __forceinline__ T warp_row_share(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                            const T* __restrict__ val, int64_t row, const T* xt, int lane,
                                            bool live, int sub, int g) {
    constexpr int SLOTS_W = 32 / W;
    const int slot = lane / W, c = lane % W;
    const int64_t e = live ? ptr[row + 1] : 0;
    const int64_t st = (int64_t)g * SLOTS_W;
    int64_t p = live ? ptr[row] + (int64_t)sub * SLOTS_W + slot : 0;
    T a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    for (; p + 3 * st < e; p += 4 * st) {
        const int32_t i0 = idx[p], i1 = idx[p + st], i2 = idx[p + 2 * st], i3 = idx[p + 3 * st];
        const T v0 = val[p], v1 = val[p + st], v2 = val[p + 2 * st], v3 = val[p + 3 * st];
        a0 += v0 * xt[(int64_t)i0 * TILE + c];
        a1 += v1 * xt[(int64_t)i1 * TILE + c];
        a2 += v2 * xt[(int64_t)i2 * TILE + c];
        a3 += v3 * xt[(int64_t)i3 * TILE + c];
    }
    for (; p < e; p += st) a0 += val[p] * xt[(int64_t)idx[p] * TILE + c];
    T acc = (a0 + a1) + (a2 + a3);
#pragma unroll
    for (int o = W; o < 32; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

// FWD: y_u = r_u - L[u, :] y (row form).  BWD: y_u = y_u / D_u (D_u != 0) - L[:, u]^T y (column form).
template <class T, bool FWD>
__device__ __forceinline__ void run_finish(const int32_t* __restrict__ rows, const T* __restrict__ aux, T* y,
                                           int64_t toff, int c, int32_t i, T acc) {
    const int64_t u = rows[i];
    const int64_t o = toff + u * TILE + c;
    if (FWD) {
        y[o] = aux[o] - acc;
    } else {
        const T d = aux[u];
        const T yu = y[o];
        y[o] = (d != (T)0 ? yu / d : yu) - acc;
    }
}

template <class T, int W, bool FWD>
__global__ void __launch_bounds__(RUN_THREADS) k_trsv_run(int64_t n, const int32_t* __restrict__ rows,
                                                          const int32_t* __restrict__ sched,
                                                          const int32_t* __restrict__ step, int32_t s0, int32_t s1,
                                                          const int64_t* __restrict__ ptr,
                                                          const int32_t* __restrict__ idx,
                                                          const T* __restrict__ val, const T* __restrict__ aux, T* y,
                                                          int32_t kcols, int nsub, RowAct ra) {
    __shared__ T s_part[RUN_WARPS][W];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t t = blockIdx.x / nsub;
    const int c0 = (int)(blockIdx.x % nsub) * W;  // first column of this block's sub-tile
    const int64_t toff = t * n * TILE;
    const bool live = t * TILE + c0 + lane % W < kcols;
    for (int32_t s = s0; s < s1; s++) {
        const int32_t a = step[s], b = step[s + 1];
        const int g = RUN_WARPS / max(1, b - a);  // warps per row
        if (g <= 1) {
            for (int32_t q = a + warp; q < b; q += RUN_WARPS) {
                const int32_t i = sched[q];
                const bool on = row_on(ra, rows[i], t);
                const T acc = warp_row_share<T, W>(ptr, idx, val, i, y + toff + c0, lane, live && on, 0, 1);
                if (lane < W && on) run_finish<T, FWD>(rows, aux, y, toff, c0 + lane, i, acc);
            }
        } else {
            const int q = warp / g, sub = warp % g;
            const bool mine = a + q < b && row_on(ra, rows[sched[a + q]], t);
            const T acc = mine ? warp_row_share<T, W>(ptr, idx, val, sched[a + q], y + toff + c0, lane, live, sub, g)
                               : (T)0;
            if (lane < W) s_part[warp][lane] = acc;
            __syncthreads();
            if (mine && sub == 0 && lane < W) {
                T tot = s_part[warp][lane];
                for (int u = 1; u < g; u++) tot += s_part[warp + u][lane];
                run_finish<T, FWD>(rows, aux, y, toff, c0 + lane, sched[a + q], tot);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- the last forward level, finished
// The rows of a factor's last level are read by no later forward level, and their columns of L are empty
// (nothing is eliminated after them; a level's rows never reference each other), so the backward solve's
// whole work on them is z_u = y_u / D_u - 0.  When the last level is a level of its own (not part of a
// thin-level run), its forward launch (M_FWD_LAST) does this too and its backward launch is skipped; each
// value is formed by the same operations in the same order as in the two launches.  At ER n = 1M the
// truncated factor's last level holds 855K of the 1M rows, and its backward launch took 5.5 ms of a 21 ms
// application.  (A kernel that gave each warp several of these short rows at once, with all their loads
// issued first, ran slower than this chunk walk: 28.8 against 20.8 ms per application.)

// ---------------------------------------------------------------- preconditioner as a CUDA graph
// values of the factor in the precision of the solve (the structure is shared)
template <class T>
struct FactorVals {
    const T* prow_val;
    const T* pcol_val;
    const T* D;
};

// Column layouts of the triangular-solve launches.  A level launch gives each warp row a width of W columns
// (8, 16 or 32; TILE / W blocks per column tile): with W = 32 a warp's lanes cover a tile's columns of one row
// (256-byte gathers); with W = 8 a warp works on four rows at once, with four times the blocks, which suits
// latency-bound levels of few rows.  Every width gives the same values bit for bit (each (row, column) sum is
// formed the same way, see k_chunked), so the width is a pure launch-shape choice: the fixed rule below, or
// widths measured level by level (tune_trsv_shapes).  Runs of thin levels always use 8 columns.  With no more
// than 8 real columns (the factor autotuner's probe) every launch uses 8 columns and one sub-tile; the padding
// columns of y must then be zero.
constexpr int NARROW_W = 8;
constexpr int SPLIT_LEVEL_ROWS = 1024;
constexpr int TRSV_NWIDTH = TILE >= 32 ? 3 : TILE >= 16 ? 2 : 1;  // widths 8, 16, 32 that fit a tile
static inline int trsv_width(int code) { return 8 << code; }

// CUDA events around each level launch of a preconditioner application (measurement only)
struct LevelEvents {
    std::vector<cudaEvent_t> ev;        // pairs: before, after
    std::vector<std::pair<bool, int32_t>> tag;  // (forward, level) of each pair
    size_t used = 0;
    ~LevelEvents() {
        for (auto e : ev) cudaEventDestroy(e);
    }
    void begin(cudaStream_t s, bool fwd, int32_t l) {
        if (2 * used == ev.size()) {
            for (int i = 0; i < 2; i++) {
                cudaEvent_t e;
                SSP_CUDA(cudaEventCreate(&e));
                ev.push_back(e);
            }
            tag.push_back({fwd, l});
        }
        tag[used] = {fwd, l};
        SSP_CUDA(cudaEventRecord(ev[2 * used], s));
    }
    void end(cudaStream_t s) {
        SSP_CUDA(cudaEventRecord(ev[2 * used + 1], s));
        used++;
    }
};

template <int MODE, class T, int MINB>
static void launch_level_w(int code, dim3 grid, cudaStream_t s, int64_t n, const int32_t* ch, int32_t nc,
                           const int64_t* ptr, const int32_t* idx, const T* val, const int32_t* rowmap, T* y,
                           const T* aux, int64_t ld, int32_t kcols, int nsub, const T* dlast, const RowAct& ra) {
    switch (code) {
    case 0:
        k_chunked<MODE, T, 8, MINB><<<grid, CH_THREADS, 0, s>>>(n, ch, nc, ptr, idx, val, rowmap, y, y, aux, ld,
                                                                nullptr, kcols, nsub, dlast, ra);
        break;
    case 1:
        k_chunked<MODE, T, (TILE >= 16 ? 16 : 8), MINB><<<grid, CH_THREADS, 0, s>>>(
            n, ch, nc, ptr, idx, val, rowmap, y, y, aux, ld, nullptr, kcols, nsub, dlast, ra);
        break;
    default:
        k_chunked<MODE, T, TILE, MINB><<<grid, CH_THREADS, 0, s>>>(n, ch, nc, ptr, idx, val, rowmap, y, y, aux, ld,
                                                                   nullptr, kcols, nsub, dlast, ra);
        break;
    }
}

// sh: per-level widths (nullptr: the fixed rule); lev: events around each level launch (nullptr: none)
template <class T>
static int64_t launch_precond(Context& C, const DevFactor& F, const FactorVals<T>& V, int64_t n, const T* r, T* y,
                              int64_t ld, int32_t kcols, const RowAct& ra = RowAct(),
                              const TrsvShapes* sh = nullptr, LevelEvents* lev = nullptr) {
    const int ntiles = (int)(ld / TILE);
    const bool narrow = TILE > NARROW_W && kcols <= NARROW_W;
    const int nsub = narrow ? 1 : TILE / NARROW_W;  // sub-tiles of the 8-column layout (runs)
    int64_t launches = 0;
    // segments in level order: the thin-level runs (by index into F.runs) and single wide levels (-1)
    std::vector<std::pair<int32_t, int32_t>> seg;  // (level, run or -1)
    for (int32_t l = 0, u = 0; l < F.num_levels;) {
        if (u < (int32_t)F.runs.size() && F.runs[u].l0 == l) {
            seg.push_back({l, u});
            l = F.runs[u++].l1;
        } else {
            seg.push_back({l++, -1});
        }
    }
    // the last level finished by its forward launch (M_FWD_LAST) when it is a level of its own;
    // SSP_PRECOND_FUSE_LAST=0 keeps the level's two launches (the same values, bit for bit; for comparisons)
    const int32_t L_last = F.num_levels - 1;
    const char* fuse_env = getenv("SSP_PRECOND_FUSE_LAST");
    const bool fuse_last = !(fuse_env && fuse_env[0] == '0') && !seg.empty() && seg.back().second < 0 &&
                           F.last_bwd_nnz == 0 && L_last >= 0;
    auto width_code = [&](bool fwd, int32_t l) -> int {
        if (narrow) return 0;
        int c = F.level_ptr[l + 1] - F.level_ptr[l] <= SPLIT_LEVEL_ROWS ? 0 : 2;
        if (sh) {
            const auto& v = fwd ? sh->fw : sh->bw;
            if ((size_t)l < v.size()) c = v[l];
        }
        return std::min(c, TRSV_NWIDTH - 1);
    };
    auto level = [&](bool fwd, int32_t l) {
        const auto& lvl = fwd ? F.fchunk_lvl : F.bchunk_lvl;
        const int32_t c0 = lvl[l], nc = lvl[l + 1] - c0;
        if (nc == 0) return;
        const int code = width_code(fwd, l);
        const int ns = narrow ? 1 : TILE / trsv_width(code);
        const dim3 grid((unsigned)chunk_blocks(nc), (unsigned)(ntiles * ns));
        const int32_t* ch = (fwd ? F.fchunk : F.bchunk) + c0;
        const bool last = fwd && fuse_last && l == L_last;
        if (lev) lev->begin(C.stream, fwd, l);
        if (last)
            launch_level_w<M_FWD_LAST, T, MINB_FWD>(code, grid, C.stream, n, ch, nc, F.prow_ptr, F.prow_idx,
                                                    V.prow_val, F.level_rows, y, r, ld, kcols, ns, V.D, ra);
        else if (fwd)
            launch_level_w<M_FWD, T, MINB_FWD>(code, grid, C.stream, n, ch, nc, F.prow_ptr, F.prow_idx, V.prow_val,
                                               F.level_rows, y, r, ld, kcols, ns, nullptr, ra);
        else
            launch_level_w<M_BWD, T, MINB_BWD>(code, grid, C.stream, n, ch, nc, F.pcol_ptr, F.pcol_idx, V.pcol_val,
                                               F.level_rows, y, V.D, ld, kcols, ns, nullptr, ra);
        if (lev) lev->end(C.stream);
        launches++;
    };
    const unsigned rgrid = (unsigned)(ntiles * nsub);
    for (size_t i = 0; i < seg.size(); i++) {
        if (seg[i].second < 0) {
            level(true, seg[i].first);
            continue;
        }
        const auto& run = F.runs[seg[i].second];
        k_trsv_run<T, NARROW_W, true><<<rgrid, RUN_THREADS, 0, C.stream>>>(
            n, F.level_rows, F.fsched, F.fstep, run.fs0, run.fs1, F.prow_ptr, F.prow_idx, V.prow_val, r, y, kcols,
            nsub, ra);
        launches++;
    }
    for (size_t i = seg.size(); i-- > 0;) {
        if (fuse_last && i + 1 == seg.size()) continue;  // finished by its forward launch (M_FWD_LAST)
        if (seg[i].second < 0) {
            level(false, seg[i].first);
            continue;
        }
        const auto& run = F.runs[seg[i].second];
        k_trsv_run<T, NARROW_W, false><<<rgrid, RUN_THREADS, 0, C.stream>>>(
            n, F.level_rows, F.bsched, F.bstep, run.bs0, run.bs1, F.pcol_ptr, F.pcol_idx, V.pcol_val, V.D, y, kcols,
            nsub, ra);
        launches++;
    }
    SSP_CHECK_LAUNCH();
    return launches;
}

// Level-launch shapes by measurement.  Each width is timed on every level launch of one preconditioner
// application (CUDA events around each launch), and each level and direction keeps its fastest width.  In a PCG
// solve the measured applications are the solve's own first three (one per width): the values are the same
// whatever the widths, so they are real iterations and nothing is applied twice; the preconditioner's graph is
// then rebuilt with the result.  The shapes are kept per context under a signature of the factor's level
// structure and the solve's shape, so repeated solves on the same graph measure once.  Small solves (n * ld
// below SSP_TRSV_TUNE_MIN elements, 2^26 unless the environment variable of that name says otherwise) keep the
// rule.  SSP_TRSV_TUNE=0 keeps the rule everywhere; SSP_TRSV_WIDTH=8|16|32 forces one width.
#ifndef SSP_TRSV_TUNE_MIN
#define SSP_TRSV_TUNE_MIN (int64_t(1) << 26)
#endif
constexpr int TRSV_CACHE_MAX = 8;
static int64_t trsv_tune_min() {
    const char* e = getenv("SSP_TRSV_TUNE_MIN");  // elements n * ld from which to measure
    return e && e[0] ? atoll(e) : (int64_t)SSP_TRSV_TUNE_MIN;
}

static uint64_t trsv_signature(const DevFactor& F, int64_t n, int64_t ld, int32_t kcols, size_t elem,
                               bool segmented) {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) {
        for (int i = 0; i < 8; i++) {
            h ^= (v >> (8 * i)) & 0xff;
            h *= 1099511628211ull;
        }
    };
    mix((uint64_t)n);
    mix((uint64_t)ld);
    mix((uint64_t)kcols);
    mix((uint64_t)elem);
    mix((uint64_t)segmented);
    // the level sizes, entry counts and runs: fixed by the factor (the order of the rows inside a level, and so
    // the chunk boundaries, may differ from one factorization to the next; the widths are chosen per level)
    mix((uint64_t)F.nnz);
    mix((uint64_t)F.num_levels);
    mix((uint64_t)F.last_fwd_nnz);
    mix((uint64_t)F.last_bwd_nnz);
    for (int32_t v : F.level_ptr) mix((uint64_t)(uint32_t)v);
    for (const auto& r : F.runs) mix(((uint64_t)(uint32_t)r.l0 << 32) | (uint32_t)r.l1);
    return h;
}

static void count_trsv_widths(const DevFactor& F, const TrsvShapes& sh, PcgReport& rep) {
    for (int i = 0; i < 3; i++) rep.trsv_levels[i] = 0;
    std::vector<bool> in_run(F.num_levels, false);
    for (const auto& r : F.runs)
        for (int32_t l = r.l0; l < r.l1; l++) in_run[l] = true;
    for (int32_t l = 0; l < F.num_levels; l++) {
        if (in_run[l]) continue;
        if (F.fchunk_lvl[l + 1] > F.fchunk_lvl[l]) rep.trsv_levels[sh.fw[l]]++;
        if (F.bchunk_lvl[l + 1] > F.bchunk_lvl[l]) rep.trsv_levels[sh.bw[l]]++;
    }
}

static int rule_code(const DevFactor& F, int32_t l, bool narrow) {
    if (narrow) return 0;
    return std::min(F.level_ptr[l + 1] - F.level_ptr[l] <= SPLIT_LEVEL_ROWS ? 0 : 2, TRSV_NWIDTH - 1);
}
static TrsvShapes rule_shapes(const DevFactor& F, bool narrow) {
    TrsvShapes s;
    s.fw.resize(F.num_levels);
    for (int32_t l = 0; l < F.num_levels; l++) s.fw[l] = (uint8_t)rule_code(F, l, narrow);
    s.bw = s.fw;
    return s;
}
static TrsvShapes forced_shapes(const DevFactor& F, int code) {
    TrsvShapes s;
    s.fw.assign(F.num_levels, (uint8_t)std::min(code, TRSV_NWIDTH - 1));
    s.bw = s.fw;
    return s;
}

// per level and direction, the width with the smallest time in ev[c] (one measured application per width
// code c); the rule's width unless another is faster
static void shapes_from_events(const DevFactor& F, const LevelEvents* ev, int nw, TrsvShapes& out) {
    const float INF = 3.0e38f;
    std::vector<float> best(2 * (size_t)F.num_levels * nw, INF);
    for (int c = 0; c < nw; c++) {
        const LevelEvents& L = ev[c];
        for (size_t i = 0; i < L.used; i++) {
            float t = 0;
            SSP_CUDA(cudaEventElapsedTime(&t, L.ev[2 * i], L.ev[2 * i + 1]));
            const size_t o = ((size_t)(L.tag[i].first ? 0 : 1) * F.num_levels + L.tag[i].second) * nw + c;
            best[o] = std::min(best[o], t);
        }
    }
    out.fw.assign(F.num_levels, 0);
    out.bw.assign(F.num_levels, 0);
    for (int dir = 0; dir < 2; dir++)
        for (int32_t l = 0; l < F.num_levels; l++) {
            const float* b = &best[((size_t)dir * F.num_levels + l) * nw];
            int pick = rule_code(F, l, false);
            for (int c = 0; c < nw; c++)
                if (b[c] < b[pick]) pick = c;
            (dir == 0 ? out.fw : out.bw)[l] = (uint8_t)pick;
        }
}

// how a solve's level shapes are chosen: Forced and Cached fill store; Measure returns the cache key
enum class ShapeSource { Rule, Forced, Cached, Measure };
static ShapeSource trsv_shape_source(Context& C, const DevFactor& F, int64_t n, int64_t ld, int32_t kcols,
                                     size_t elem, bool segmented, TrsvShapes& store, uint64_t& key) {
    const bool narrow = TILE > NARROW_W && kcols <= NARROW_W;
    if (narrow || F.num_levels == 0) return ShapeSource::Rule;  // one width for all (8 columns)
    const char* fw = getenv("SSP_TRSV_WIDTH");
    if (fw && fw[0]) {
        const int w = atoi(fw);
        store = forced_shapes(F, w >= 32 ? 2 : w >= 16 ? 1 : 0);
        return ShapeSource::Forced;
    }
    const char* tn = getenv("SSP_TRSV_TUNE");
    if ((tn && tn[0] == '0') || n * ld < trsv_tune_min()) return ShapeSource::Rule;
    key = trsv_signature(F, n, ld, kcols, elem, segmented);
    for (auto& e : C.trsv_cache.entries)
        if (e.first == key) {
            store = e.second;
            return ShapeSource::Cached;
        }
    return ShapeSource::Measure;
}

static void cache_shapes(Context& C, uint64_t key, const TrsvShapes& s) {
    auto& E = C.trsv_cache.entries;
    if ((int)E.size() >= TRSV_CACHE_MAX) E.erase(E.begin());
    E.push_back({key, s});
}

static void report_shapes(PcgReport& rep, int32_t source, const DevFactor& F, const TrsvShapes& s) {
    rep.trsv_shapes = source;
    count_trsv_widths(F, s, rep);
}

// Three applications, one per width, then the per-level choice (the stage entry point's measurement).
template <class T>
static void tune_trsv_shapes(Context& C, const DevFactor& F, const FactorVals<T>& V, int64_t n, const T* r, T* y,
                             int64_t ld, int32_t kcols, const RowAct& ra, TrsvShapes& out) {
    LevelEvents ev[3];
    for (int c = 0; c < TRSV_NWIDTH; c++) {
        const TrsvShapes f = forced_shapes(F, c);
        C.kernels_launched += launch_precond<T>(C, F, V, n, r, y, ld, kcols, ra, &f, &ev[c]);
    }
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    shapes_from_events(F, ev, TRSV_NWIDTH, out);
}

// The preconditioner application as a CUDA graph, with its level shapes.  measure: the shapes are still to be
// measured by the solve's next applications (pcg_solve), which then rebuild the graph.
struct Precond {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    TrsvShapes shapes;
    bool has_shapes = false;
    bool measure = false;
    uint64_t key = 0;
    int mstep = 0;                 // widths measured so far
    LevelEvents mev[3];            // their level launches
    cudaEvent_t m0 = nullptr, m1 = nullptr;  // around the measured applications
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    ~Precond() {
        drop_graph();
        if (m0) cudaEventDestroy(m0);
        if (m1) cudaEventDestroy(m1);
    }
};

// ---------------------------------------------------------------- SpMM plan
// The Laplacian as the SpMM reads it.  When one tile of the gathered operand (n rows of TILE values) is
// far larger than L2 and the matrix has no locality to exploit (random graphs: a row's neighbours are
// anywhere), the columns are cut into nslabs equal ranges and the entries stored slab-major: slab b,
// row i holds row i's entries with a column in slab b, in their stored order, at ptr[b n + i] ..
// ptr[b n + i + 1].  The SpMM then makes one pass per slab (the first writes q, the others add into it),
// and each pass gathers from a 1/nslabs share of the tile that stays resident in L2; the price is
// 2 nslabs - 1 streaming passes over q instead of 1.  Measured on B200 (ER n = 1M, average degree 20,
// 1327 columns, FP64): one pass 39.5 ms; 3, 4, 6, 8, 11 slabs 48.0, 52.6, 63.4, 75.4, 93.7 ms -- the extra q
// passes cost more than the L2 hits save, so slabs are off unless SSP_SPMM_SLAB_MB (the L2 share of one
// slab, MB) asks for them.
constexpr int MAX_SLABS = 16;

double spmm_slab_mb() {
    const char* e = getenv("SSP_SPMM_SLAB_MB");
    return e ? atof(e) : 0.0;
}

struct SpmmPlan {
    int32_t nslabs = 1;
    int64_t nnz = 0;
    const int64_t* ptr = nullptr;  // nslabs * n + 1 row pointers
    const int32_t* idx = nullptr;
    const double* val = nullptr;  // FP64 values in this entry order
    const int32_t* chunks[MAX_SLABS] = {};
    int32_t nchunks[MAX_SLABS] = {};
    dim3 grid;
    double* part = nullptr;
};

// entries farther than `window` from the diagonal, summed per block into *far
__global__ void k_far_count(int64_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                            int64_t window, unsigned long long* far) {
    __shared__ unsigned long long s_far;
    if (threadIdx.x == 0) s_far = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    unsigned c = 0;
    if (i < n)
        for (int64_t e = ptr[i] + lane; e < ptr[i + 1]; e += 32) c += llabs((int64_t)idx[e] - i) > window;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0 && c) atomicAdd(&s_far, (unsigned long long)c);
    __syncthreads();
    if (threadIdx.x == 0 && s_far) atomicAdd(far, s_far);
}

// per (slab, row) entry counts; one warp per row, lane b keeps slab b's count
__global__ void k_slab_count(int64_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                             int64_t slab_rows, int32_t nslabs, int32_t* __restrict__ cnt) {
    const int lane = threadIdx.x & 31;
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= n) return;
    int32_t mine = 0;
    for (int64_t e0 = ptr[i]; e0 < ptr[i + 1]; e0 += 32) {
        const int64_t e = e0 + lane;
        const int b = e < ptr[i + 1] ? (int)(idx[e] / slab_rows) : -1;
        for (int s = 0; s < nslabs; s++) {
            const int c = __popc(__ballot_sync(0xffffffffu, b == s));
            if (lane == s) mine += c;
        }
    }
    if (lane < nslabs) cnt[(int64_t)lane * n + i] = mine;
}

// stable partition of each row's entries into the slab-major copy
__global__ void k_slab_fill(int64_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                            const double* __restrict__ val, int64_t slab_rows, int32_t nslabs,
                            const int64_t* __restrict__ sptr, int32_t* __restrict__ sidx,
                            double* __restrict__ sval) {
    const int lane = threadIdx.x & 31;
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= n) return;
    int64_t base = lane < nslabs ? sptr[(int64_t)lane * n + i] : 0;  // lane b: next free slot of slab b
    const unsigned lt = (1u << lane) - 1u;
    for (int64_t e0 = ptr[i]; e0 < ptr[i + 1]; e0 += 32) {
        const int64_t e = e0 + lane;
        const bool in = e < ptr[i + 1];
        const int b = in ? (int)(idx[e] / slab_rows) : -1;
        for (int s = 0; s < nslabs; s++) {
            const unsigned bal = __ballot_sync(0xffffffffu, b == s);
            const int64_t at = __shfl_sync(0xffffffffu, base, s);
            if (b == s) {
                const int64_t pos = at + __popc(bal & lt);
                sidx[pos] = idx[e];
                sval[pos] = val[e];
            }
            if (lane == s) base += __popc(bal);
        }
    }
}

static int32_t spmm_slab_count(Context& C, int64_t n, const int64_t* ptr, const int32_t* idx, int64_t nnz) {
    const double mb = spmm_slab_mb();
    if (!(mb > 0) || nnz == 0) return 1;
    // slabs are cut for the FP64 operand (TILE doubles per row); FP32 solves use the same cut
    const int64_t slab_rows = std::max<int64_t>(1, (int64_t)(mb * 1048576.0 / (TILE * sizeof(double))));
    if (n <= slab_rows) return 1;
    unsigned long long* far = C.ws.get_t<unsigned long long>("pcg_slab_far", 1);
    SSP_CUDA(cudaMemsetAsync(far, 0, sizeof(unsigned long long), C.stream));
    k_far_count<<<(unsigned)ceil_div<int64_t>(n * 32, 256), 256, 0, C.stream>>>(n, ptr, idx, slab_rows / 2, far);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    // a matrix whose entries mostly sit near the diagonal already reuses L2 in a row sweep
    if (read_i64(C, reinterpret_cast<const int64_t*>(far)) * 4 < nnz) return 1;
    return (int32_t)std::min<int64_t>(MAX_SLABS, ceil_div<int64_t>(n, slab_rows));
}

static SpmmPlan make_spmm_plan(Context& C, int64_t n, const int64_t* lap_ptr, const int32_t* lap_idx,
                               const double* lap_val, int64_t ld) {
    Workspace& W = C.ws;
    SpmmPlan A;
    A.nnz = read_i64(C, lap_ptr + n);
    A.nslabs = spmm_slab_count(C, n, lap_ptr, lap_idx, A.nnz);
    const int32_t m = A.nslabs;
    std::vector<int64_t> hp((size_t)m * n + 1);
    if (m == 1) {
        A.ptr = lap_ptr;
        A.idx = lap_idx;
        A.val = lap_val;
    } else {
        const int64_t slab_rows = ceil_div<int64_t>(n, m);
        int32_t* cnt = W.get_t<int32_t>("pcg_slab_cnt", (size_t)m * n);
        int64_t* sptr = W.get_t<int64_t>("pcg_slab_ptr", (size_t)m * n + 1);
        int32_t* sidx = W.get_t<int32_t>("pcg_slab_idx", A.nnz + 1);
        double* sval = W.get_t<double>("pcg_slab_val", A.nnz + 1);
        const unsigned blocks = (unsigned)ceil_div<int64_t>(n * 32, 256);
        k_slab_count<<<blocks, 256, 0, C.stream>>>(n, lap_ptr, lap_idx, slab_rows, m, cnt);
        SSP_CHECK_LAUNCH();
        exclusive_scan_i32_to_i64(C, cnt, sptr, (int64_t)m * n, sptr + (int64_t)m * n);
        k_slab_fill<<<blocks, 256, 0, C.stream>>>(n, lap_ptr, lap_idx, lap_val, slab_rows, m, sptr, sidx, sval);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += 2;
        A.ptr = sptr;
        A.idx = sidx;
        A.val = sval;
    }
    SSP_CUDA(cudaMemcpyAsync(hp.data(), A.ptr, sizeof(int64_t) * hp.size(), cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    std::vector<int32_t> all;
    std::vector<size_t> off(m);
    int32_t most = 0;
    for (int32_t b = 0; b < m; b++) {
        off[b] = all.size();
        const size_t before = all.size();
        make_chunks(hp.data() + (size_t)b * n, 0, (int32_t)n, all);
        A.nchunks[b] = (int32_t)(all.size() - before);
        most = std::max(most, A.nchunks[b]);
        all.push_back((int32_t)n);
    }
    int32_t* d = W.get_t<int32_t>("pcg_achunks", all.size());
    SSP_CUDA(cudaMemcpyAsync(d, all.data(), sizeof(int32_t) * all.size(), cudaMemcpyHostToDevice, C.stream));
    for (int32_t b = 0; b < m; b++) A.chunks[b] = d + off[b];
    const int bx = chunk_blocks(most);
    A.grid = dim3((unsigned)bx, (unsigned)(ld / TILE));
    A.part = W.get_t<double>("pcg_spmm_part", (size_t)bx * ld);
    return A;
}

// SpMM q = A p over the plan's slabs (+ p.q partials into A.part when dot)
template <class T>
static void launch_spmm(Context& C, int64_t n, const SpmmPlan& A, const T* aval, const T* p, T* q, int64_t ld,
                        bool dot, int32_t kcols, const RowAct& ra = RowAct()) {
    const bool narrow = TILE > NARROW_W && kcols <= NARROW_W;
    for (int32_t b = 0; b < A.nslabs; b++) {
        const int64_t* ptr = A.ptr + (int64_t)b * n;
        double* part = dot && b == A.nslabs - 1 ? A.part : nullptr;
#define SSP_SPMM_LAUNCH(MODE, W_)                                                                                  \
    k_chunked<MODE, T, W_, MINB_SPMM><<<A.grid, CH_THREADS, 0, C.stream>>>(n, A.chunks[b], A.nchunks[b], ptr, A.idx,  \
                                                                            aval, nullptr, p, q, nullptr, ld, part,    \
                                                                            kcols, 1, nullptr, ra)
        if (b == 0) {
            if (narrow) SSP_SPMM_LAUNCH(M_SPMM, NARROW_W);
            else SSP_SPMM_LAUNCH(M_SPMM, TILE);
        } else {
            if (narrow) SSP_SPMM_LAUNCH(M_SPMM_ACC, NARROW_W);
            else SSP_SPMM_LAUNCH(M_SPMM_ACC, TILE);
        }
#undef SSP_SPMM_LAUNCH
    }
}

// One preconditioner application from the solve's r into its z with the given level shapes (nullptr: the rule)
// and optional events around each level launch; returns the kernels it launched.
using PcApply = std::function<int64_t(const TrsvShapes*, LevelEvents*)>;

// P's graph: one application with P's shapes (the rule when it has none)
static void capture_precond(Context& C, Precond& P, int64_t& launches, const PcApply& pc) {
    P.drop_graph();
    SSP_CUDA(cudaStreamBeginCapture(C.stream, cudaStreamCaptureModeThreadLocal));
    try {
        launches = pc(P.has_shapes ? &P.shapes : nullptr, nullptr);
    } catch (...) {
        cudaGraph_t g;
        cudaStreamEndCapture(C.stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    SSP_CUDA(cudaStreamEndCapture(C.stream, &P.graph));
    SSP_CUDA(cudaGraphInstantiate(&P.exec, P.graph, 0));
}

// The solve's preconditioner: its level shapes (forced, cached, the rule, or the rule until the solve's first
// applications have measured them) and its graph.  elem: bytes per value of the triangular solves.
static void build_precond_graph(Context& C, const DevFactor& F, int64_t n, int64_t ld, int32_t kcols, size_t elem,
                                Precond& P, int64_t& launches, PcgReport& rep, const RowAct& ra,
                                const PcApply& pc) {
    TrsvShapes store;
    uint64_t key = 0;
    const bool narrow = TILE > NARROW_W && kcols <= NARROW_W;
    const ShapeSource src = trsv_shape_source(C, F, n, ld, kcols, elem, ra.act != nullptr, store, key);
    P.measure = false;
    P.has_shapes = src == ShapeSource::Forced || src == ShapeSource::Cached;
    if (P.has_shapes) {
        P.shapes = store;
        report_shapes(rep, src == ShapeSource::Forced ? SSP_TRSV_FORCED : SSP_TRSV_CACHED, F, store);
    } else {
        report_shapes(rep, SSP_TRSV_RULE, F, rule_shapes(F, narrow));
        if (src == ShapeSource::Measure) {
            P.measure = true;
            P.key = key;
            P.mstep = 0;
        }
    }
    capture_precond(C, P, launches, pc);
}

static FactorVals<double> fp64_vals(const DevFactor& F) { return FactorVals<double>{F.prow_val, F.pcol_val, F.D}; }

// apply M^{-1} to R into Z once (tile-major n x ld blocks; stage entry point).  When the shapes are to be
// measured, one application per width measures them first (each writes the same Z).
void precond_apply_device(Context& C, const DevFactor& F, const double* R, double* Z, int64_t ld) {
    TrsvShapes store;
    uint64_t key = 0;
    const ShapeSource src = trsv_shape_source(C, F, F.n, ld, (int32_t)ld, sizeof(double), false, store, key);
    const TrsvShapes* sh = nullptr;
    if (src == ShapeSource::Forced || src == ShapeSource::Cached) {
        sh = &store;
    } else if (src == ShapeSource::Measure) {
        tune_trsv_shapes<double>(C, F, fp64_vals(F), F.n, R, Z, ld, (int32_t)ld, RowAct(), store);
        cache_shapes(C, key, store);
        sh = &store;
    }
    int64_t l = launch_precond<double>(C, F, fp64_vals(F), F.n, R, Z, ld, (int32_t)ld, RowAct(), sh);
    C.kernels_launched += l;
}

// ---------------------------------------------------------------- per-kernel event timing
struct EventPairs {
    std::vector<cudaEvent_t> a, b;
    size_t used = 0;
    ~EventPairs() {
        for (auto e : a) cudaEventDestroy(e);
        for (auto e : b) cudaEventDestroy(e);
    }
    void begin(cudaStream_t s) {
        if (used == a.size()) {
            cudaEvent_t x, y;
            SSP_CUDA(cudaEventCreate(&x));
            SSP_CUDA(cudaEventCreate(&y));
            a.push_back(x);
            b.push_back(y);
        }
        SSP_CUDA(cudaEventRecord(a[used], s));
    }
    void end(cudaStream_t s) { SSP_CUDA(cudaEventRecord(b[used++], s)); }
    double total_ms() {
        double t = 0;
        for (size_t i = 0; i < used; i++) {
            float x = 0;
            cudaEventElapsedTime(&x, a[i], b[i]);
            t += x;
        }
        return t;
    }
};

// ---------------------------------------------------------------- one PCG solve in one precision
template <class T>
struct PcgBufs {
    T* e;  // solution increment (zero on entry)
    T* r;  // right-hand side on entry, residual on exit
    T* z;
    T* p;
    T* q;
};

struct PcgTimers {
    EventPairs spmm, pc, loop;
};

// Runs PCG on A e = r for every column that S marks active (S.thr, S.active, S.nactive set by the
// caller; e zero).  Returns the iterations of the loop.
template <class T>
static int32_t pcg_solve(Context& C, int64_t n, int32_t k, int64_t ld, const SpmmPlan& A, const T* aval,
                         const DevFactor& F, const PcApply& pc,
                         Precond& P, int64_t& pc_launches, PcgBufs<T> B, ColState& S, Reducer& R,
                         int32_t max_iters, const PcgOptions& opt, PcgTimers& tm, PcgReport& rep,
                         const RowAct& ra = RowAct()) {
    // without a residual history or progress output the iterations after the first run on the device
    // SSP_PCG_HOST_LOOP=1 keeps every iteration on the host loop (the same kernels, launched one by one), for
    // profilers that do not look inside conditional graph nodes
    static const bool host_loop = [] {
        const char* e = getenv("SSP_PCG_HOST_LOOP");
        return e && e[0] == '1';
    }();
    const bool seg_history = opt.segs && opt.segs->record_history;
    const bool device_loop = !opt.history && !seg_history && !opt.verbose && !host_loop;
    const int64_t ntiles = ld / TILE;
    const int64_t total = n * ld;
    const dim3 egrid((unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div<int64_t>(n * TILE, 256),
                                                                      2048 / std::max<int64_t>(1, ntiles) + 4)),
                     (unsigned)ntiles);
    const SegDev& G = R.G;
    const int64_t ns = (int64_t)G.nseg * ld;  // per-(graph, column) state entries
    const int cg = grid_for(ns, 256);
    // with several graphs the SpMM's blocks straddle graphs, so p.q is a segmented reduction of its own
    auto pq_dot = [&]() {
        if (G.nseg > 1) R.run<OP_DOT, T>(B.p, B.q, S.pq);
        else colred_final(C, ld, (int)A.grid.x, A.part, S.pq);
    };
    // which (graph, tile) pairs still have an active column: the row kernels skip the others
    auto update_act = [&]() {
        if (!ra.act) return;
        k_seg_tile_active<<<grid_for((int64_t)G.nseg * ntiles, 256), 256, 0, C.stream>>>(G.nseg, (int32_t)ntiles, ld,
                                                                                        S.active, (int32_t*)ra.act);
        C.kernels_launched++;
    };
    // one preconditioner application: the graph, or while the level shapes are being measured, one width's
    // launches with events around each level (a real application: every width gives the same values)
    auto apply_precond = [&]() {
        tm.pc.begin(C.stream);
        if (P.measure && P.mstep < TRSV_NWIDTH) {
            if (P.mstep == 0) {
                if (!P.m0) SSP_CUDA(cudaEventCreate(&P.m0));
                if (!P.m1) SSP_CUDA(cudaEventCreate(&P.m1));
                SSP_CUDA(cudaEventRecord(P.m0, C.stream));
            }
            const TrsvShapes f = forced_shapes(F, P.mstep);
            C.kernels_launched += pc(&f, &P.mev[P.mstep]);
            if (++P.mstep == TRSV_NWIDTH) SSP_CUDA(cudaEventRecord(P.m1, C.stream));
        } else {
            SSP_CUDA(cudaGraphLaunch(P.exec, C.stream));
            C.kernels_launched += pc_launches;
        }
        tm.pc.end(C.stream);
    };
    // after a synchronization that follows the last measured application: keep the fastest width per level,
    // cache it, and rebuild the graph with it
    auto finish_measure = [&]() {
        if (!P.measure || P.mstep < TRSV_NWIDTH) return;
        shapes_from_events(F, P.mev, TRSV_NWIDTH, P.shapes);
        float ms = 0;
        SSP_CUDA(cudaEventElapsedTime(&ms, P.m0, P.m1));
        rep.ms_trsv_tune += ms;
        P.has_shapes = true;
        P.measure = false;
        cache_shapes(C, P.key, P.shapes);
        report_shapes(rep, SSP_TRSV_TUNED, F, P.shapes);
        capture_precond(C, P, pc_launches, pc);
    };
    int64_t active = read_i64(C, S.nactive);
    int32_t it = 0;
    if (active == 0) return 0;
    update_act();
    apply_precond();
    R.run<OP_DOT, T>(B.r, B.z, S.rz);
    SSP_CUDA(cudaMemcpyAsync(B.p, B.z, sizeof(T) * total, cudaMemcpyDeviceToDevice, C.stream));
    tm.loop.begin(C.stream);
    while (it < max_iters) {
        tm.spmm.begin(C.stream);
        launch_spmm<T>(C, n, A, aval, B.p, B.q, ld, G.nseg == 1, k, ra);
        tm.spmm.end(C.stream);
        pq_dot();
        k_cols_alpha<<<cg, 256, 0, C.stream>>>(ns, S);
        k_axpy_r_rr<T><<<dim3((unsigned)R.nparts, (unsigned)ntiles), RED_THREADS, 0, C.stream>>>(
            n, S.alpha, B.q, B.r, R.rows_per_blk, ld, R.part, G);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += 3 + A.nslabs;
        R.finish(S.rr);
        it++;
        SSP_CUDA(cudaMemsetAsync(S.nactive, 0, sizeof(int64_t), C.stream));
        k_cols_check<<<cg, 256, 0, C.stream>>>(ns, it, S);
        SSP_CHECK_LAUNCH();
        C.kernels_launched++;
        update_act();
        active = read_i64(C, S.nactive);
        finish_measure();
        if (opt.history || seg_history) {
            std::vector<double> hrr(ns), hbb(ns);
            SSP_CUDA(cudaMemcpyAsync(hrr.data(), S.rr, sizeof(double) * ns, cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaMemcpyAsync(hbb.data(), S.bnorm2, sizeof(double) * ns, cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaStreamSynchronize(C.stream));
            double mx = 0.0;
            for (int64_t j = 0; j < ns; j++)
                if (hbb[j] > 0) mx = std::max(mx, std::sqrt(hrr[j] / hbb[j]));
            if (opt.history) opt.history->push_back(mx);
            if (seg_history) {
                auto& H = opt.segs->history;
                H.resize(G.nseg);
                for (int32_t sg = 0; sg < G.nseg; sg++) {
                    double m2 = 0.0;
                    for (int64_t j = 0; j < ld; j++) {
                        const int64_t o = (int64_t)sg * ld + j;
                        if (hbb[o] > 0) m2 = std::max(m2, std::sqrt(hrr[o] / hbb[o]));
                    }
                    H[sg].push_back(m2);
                }
            }
        }
        if (opt.verbose && (it % 10 == 0 || active == 0))
            fprintf(stderr, "[ssp] pcg%s iter %d: %lld columns active\n", sizeof(T) == 4 ? " (fp32 inner)" : "", it,
                    (long long)active);
        if (active == 0) break;
        if (device_loop && !P.measure) break;
        apply_precond();
        R.run<OP_DOT, T>(B.r, B.z, S.rz_new);
        k_cols_beta<<<cg, 256, 0, C.stream>>>(ns, S);
        k_update_xp<T><<<egrid, 256, 0, C.stream>>>(n, ld, S.alpha, S.beta, B.z, B.p, B.e, G);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += 2;
    }
    if (device_loop && active > 0 && it < max_iters) {
        // one iteration = preconditioner, r.z, beta, p update, SpMM, alpha, x/r update, check, control
        int32_t* d_it = C.ws.get_t<int32_t>("pcg_loop_it", 1);
        k_it_set<<<1, 1, 0, C.stream>>>(d_it, it);
        SSP_CHECK_LAUNCH();
        LoopGraph L;
        cudaGraphConditionalHandle h;
        const int64_t k_before = C.kernels_launched;
        int64_t body_kernels = 0;
        SSP_CUDA(cudaGraphCreate(&L.graph, 0));
        SSP_CUDA(cudaGraphConditionalHandleCreate(&h, L.graph, 0, cudaGraphCondAssignDefault));
        auto capture = [&](cudaGraph_t g, auto&& fn) {
            SSP_CUDA(cudaStreamBeginCaptureToGraph(C.stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            try {
                fn();
            } catch (...) {
                cudaGraph_t tmp;
                cudaStreamEndCapture(C.stream, &tmp);
                throw;
            }
            SSP_CUDA(cudaStreamEndCapture(C.stream, &g));
        };
        capture(L.graph, [&] {
            k_loop_ctl<<<1, 1, 0, C.stream>>>(h, S.nactive, d_it, max_iters);
            SSP_CHECK_LAUNCH();
        });
        size_t nn = 0;
        SSP_CUDA(cudaGraphGetNodes(L.graph, nullptr, &nn));
        std::vector<cudaGraphNode_t> roots(nn);
        SSP_CUDA(cudaGraphGetNodes(L.graph, roots.data(), &nn));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t wnode;
        SSP_CUDA(cudaGraphAddNode(&wnode, L.graph, roots.data(), nn, &cp));
        capture(cp.conditional.phGraph_out[0], [&] {
            body_kernels += pc(P.has_shapes ? &P.shapes : nullptr, nullptr);
            R.run<OP_DOT, T>(B.r, B.z, S.rz_new);
            k_cols_beta<<<cg, 256, 0, C.stream>>>(ns, S);
            k_update_xp<T><<<egrid, 256, 0, C.stream>>>(n, ld, S.alpha, S.beta, B.z, B.p, B.e, G);
            launch_spmm<T>(C, n, A, aval, B.p, B.q, ld, G.nseg == 1, k, ra);
            pq_dot();
            k_cols_alpha<<<cg, 256, 0, C.stream>>>(ns, S);
            k_axpy_r_rr<T><<<dim3((unsigned)R.nparts, (unsigned)ntiles), RED_THREADS, 0, C.stream>>>(
                n, S.alpha, B.q, B.r, R.rows_per_blk, ld, R.part, G);
            R.finish(S.rr);
            k_it_next<<<1, 1, 0, C.stream>>>(d_it);
            SSP_CUDA(cudaMemsetAsync(S.nactive, 0, sizeof(int64_t), C.stream));
            k_cols_check_at<<<cg, 256, 0, C.stream>>>(ns, d_it, S);
            update_act();
            k_loop_ctl<<<1, 1, 0, C.stream>>>(h, S.nactive, d_it, max_iters);
            SSP_CHECK_LAUNCH();
        });
        // the helpers count theirs; with several graphs p.q is a reduction (counted) instead of a final pass
        body_kernels += (C.kernels_launched - k_before) + 9 + A.nslabs - (G.nseg > 1 ? 1 : 0);
        C.kernels_launched = k_before;
        SSP_CUDA(cudaGraphInstantiate(&L.exec, L.graph, 0));
        SSP_CUDA(cudaGraphLaunch(L.exec, C.stream));
        int32_t it_end = it;
        SSP_CUDA(cudaMemcpyAsync(&it_end, d_it, sizeof(int32_t), cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
        C.kernels_launched += 1 + body_kernels * (int64_t)(it_end - it);
        it = it_end;
    }
    // the last step's x += alpha p (alpha is 0 for columns that stopped earlier)
    k_axpy_x<T><<<egrid, 256, 0, C.stream>>>(n, ld, S.alpha, B.p, B.e, G);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    tm.loop.end(C.stream);
    return it;
}

// ---------------------------------------------------------------- driver
// Y: tile-major n x ld (ld = round8(k)), read only.  The solution stays in the workspace buffer
// "pcg_x" (tile-major); *x_out points at it.
void pcg_device(Context& C, int64_t n, const int64_t* lap_ptr, const int32_t* lap_idx, const double* lap_val,
                const DevFactor& F, const double* Y, int32_t k, const double** x_out, const PcgOptions& opt,
                PcgReport& rep, int32_t* h_iters, double* h_relres, const int32_t* lap_eid, double* d2,
                bool d2_accumulate) {
    SSP_REQUIRE(k > 0, SSP_ERR_INVALID, "pcg: k must be positive");
    const bool mixed = opt.precision == SSP_PRECISION_MIXED;
    SSP_REQUIRE(mixed || opt.precision == SSP_PRECISION_FP64 || opt.precision == SSP_PRECISION_PC32, SSP_ERR_INVALID,
                "pcg: unknown precision");
    const int64_t ld = ((int64_t)k + TILE - 1) / TILE * TILE;
    const int64_t ntiles = ld / TILE;
    const int64_t total = n * ld;
    Workspace& W = C.ws;
    double* x = W.get_t<double>("pcg_x", total);
    double* r = W.get_t<double>("pcg_r", total);
    double* z = W.get_t<double>("pcg_z", total);
    double* p = W.get_t<double>("pcg_p", total);
    double* q = W.get_t<double>("pcg_q", total);
    // graphs solved at once (one segment: a single graph)
    SegDev G;
    PcgSegments* segs = opt.segs;
    if (segs) {
        const int32_t nseg = (int32_t)segs->k.size();
        SSP_REQUIRE(nseg >= 1 && (int64_t)segs->row0.size() == nseg + 1 && segs->row0.front() == 0 &&
                        segs->row0.back() == n && segs->rowseg,
                    SSP_ERR_INVALID, "pcg: inconsistent graph segments");
        std::vector<int64_t> rows(nseg);
        for (int32_t i = 0; i < nseg; i++) {
            SSP_REQUIRE(segs->k[i] >= 1 && segs->k[i] <= k && segs->row0[i + 1] > segs->row0[i], SSP_ERR_INVALID,
                        "pcg: a graph segment needs rows and 1..k columns");
            rows[i] = segs->row0[i + 1] - segs->row0[i];
        }
        int32_t* d_k = W.get_t<int32_t>("pcg_seg_k", nseg);
        int64_t* d_rows = W.get_t<int64_t>("pcg_seg_rows", nseg);
        SSP_CUDA(cudaMemcpyAsync(d_k, segs->k.data(), sizeof(int32_t) * nseg, cudaMemcpyHostToDevice, C.stream));
        SSP_CUDA(cudaMemcpyAsync(d_rows, rows.data(), sizeof(int64_t) * nseg, cudaMemcpyHostToDevice, C.stream));
        G.nseg = nseg;
        G.rowseg = segs->rowseg;
        G.kseg = d_k;
        G.segrows = d_rows;
    }
    const int64_t ns = (int64_t)G.nseg * ld;  // per-(graph, column) state entries
    ColState S = make_colstate(C, ns, "pcg");
    double* colv = W.get_t<double>("pcg_aux", 3 * ns);
    double* colsum = colv;
    double* relres = colv + ns;
    double* mean = colv + 2 * ns;
    Reducer R;
    R.init(C, n, ld, "pcg_red_part", G, segs ? &segs->row0 : nullptr);
    // SpMM: row-aligned chunks of the Laplacian (column slabs on large random graphs), about one wave of
    // blocks per tile
    const SpmmPlan A = make_spmm_plan(C, n, lap_ptr, lap_idx, lap_val, ld);
    const int64_t lap_nnz = A.nnz;
    const dim3 egrid((unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div<int64_t>(n * TILE, 256),
                                                                      2048 / std::max<int64_t>(1, ntiles) + 4)),
                     (unsigned)ntiles);
    const int cg = grid_for(ns, 256);
    RowAct ra;
    if (G.nseg > 1) {
        ra.act = W.get_t<int32_t>("pcg_act", (size_t)G.nseg * ntiles);
        ra.rowseg = G.rowseg;
        ra.ntiles = (int32_t)ntiles;
    }

    // r = Y - mean(Y); x = 0; ||b||^2
    R.run<OP_SUM, double>(Y, nullptr, colsum);
    k_center<<<egrid, 256, 0, C.stream>>>(n, k, ld, Y, colsum, r, x, mean, R.G);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    R.run<OP_SQ, double>(r, nullptr, S.bnorm2);
    SSP_CUDA(cudaMemsetAsync(S.nactive, 0, sizeof(int64_t), C.stream));
    k_cols_init<<<cg, 256, 0, C.stream>>>(ld, k, opt.tol, opt.abs_tol, S, R.G);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;

    // a narrow solve leaves the padding columns of its gathered outputs untouched: start them at zero
    if (TILE > NARROW_W && k <= NARROW_W) {
        SSP_CUDA(cudaMemsetAsync(z, 0, sizeof(double) * total, C.stream));
        SSP_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * total, C.stream));
        SSP_CUDA(cudaMemsetAsync(q, 0, sizeof(double) * total, C.stream));
    }
    PcgTimers tm;
    EventPairs ev_resid;
    int32_t it = 0;
    rep = PcgReport();
    if (!mixed) {
        Precond P;
        int64_t pc_launches = 0;
        if (read_i64(C, S.nactive) > 0) {
            PcApply pc;
            size_t elem = sizeof(double);
            if (opt.precision == SSP_PRECISION_PC32 && !(TILE > NARROW_W && k <= NARROW_W)) {
                // FP64 PCG with the triangular solves in FP32: r rounded on the way in, z widened on the way out
                float* fv = W.get_t<float>("pcgp_fval", 2 * F.nnz + n + 1);
                const int64_t fcount[3] = {F.nnz, F.nnz, n};
                const double* fsrc[3] = {F.prow_val, F.pcol_val, F.D};
                int64_t at = 0;
                for (int i = 0; i < 3; i++) {
                    if (fcount[i] > 0)
                        k_d2f<<<grid_for(fcount[i], 256, 148 * 16), 256, 0, C.stream>>>(fcount[i], fsrc[i], fv + at);
                    at += fcount[i];
                }
                SSP_CHECK_LAUNCH();
                C.kernels_launched += 3;
                const FactorVals<float> V32{fv, fv + F.nnz, fv + 2 * F.nnz};
                // r32 and z32 live in q's memory: q (= A p) is dead from the r update to the next Laplacian
                // product, and the preconditioner runs in between, so this mode needs no more memory than FP64
                float* r32 = reinterpret_cast<float*>(q);
                float* z32 = r32 + total;
                const int cgrid = grid_for(total, 256, 148 * 16);
                pc = [&C, &F, V32, n, r32, z32, r, z, ld, k, ra, total, cgrid](const TrsvShapes* sh, LevelEvents* lev) {
                    k_d2f<<<cgrid, 256, 0, C.stream>>>(total, r, r32);
                    const int64_t l = launch_precond<float>(C, F, V32, n, r32, z32, ld, k, ra, sh, lev);
                    k_f2d<<<cgrid, 256, 0, C.stream>>>(total, z32, z);
                    SSP_CHECK_LAUNCH();
                    return l + 2;
                };
                elem = sizeof(float);
            } else {
                pc = [&C, &F, n, r, z, ld, k, ra](const TrsvShapes* sh, LevelEvents* lev) {
                    return launch_precond<double>(C, F, fp64_vals(F), n, r, z, ld, k, ra, sh, lev);
                };
            }
            build_precond_graph(C, F, n, ld, k, elem, P, pc_launches, rep, ra, pc);
            it = pcg_solve<double>(C, n, k, ld, A, A.val, F, pc, P, pc_launches,
                                   PcgBufs<double>{x, r, z, p, q}, S, R, opt.max_iters, opt, tm, rep, ra);
        }
    } else {
        // FP32 copies of the Laplacian and factor values, and the FP32 inner vectors
        float* aval32 = W.get_t<float>("pcgm_aval", lap_nnz + 1);
        float* fval32 = W.get_t<float>("pcgm_fval", 2 * F.nnz + n + 1);
        auto to_f32 = [&](int64_t count, const double* src, float* dst) {
            if (count <= 0) return;
            k_d2f<<<grid_for(count, 256, 148 * 16), 256, 0, C.stream>>>(count, src, dst);
            SSP_CHECK_LAUNCH();
            C.kernels_launched++;
        };
        to_f32(lap_nnz, A.val, aval32);
        to_f32(F.nnz, F.prow_val, fval32);
        to_f32(F.nnz, F.pcol_val, fval32 + F.nnz);
        to_f32(n, F.D, fval32 + 2 * F.nnz);
        const FactorVals<float> V32{fval32, fval32 + F.nnz, fval32 + 2 * F.nnz};
        float* e32 = W.get_t<float>("pcgm_e", total);
        float* r32 = W.get_t<float>("pcgm_r", total);
        float* z32 = W.get_t<float>("pcgm_z", total);
        float* p32 = W.get_t<float>("pcgm_p", total);
        float* q32 = W.get_t<float>("pcgm_q", total);
        ColState Si = make_colstate(C, ns, "pcgm_in");
        double* worst = W.get_t<double>("pcgm_worst", 1);
        double* e64 = nullptr;  // FP64 inner increment, only if a round falls back
        Precond P32, P64;
        int64_t pc32 = 0, pc64 = 0;
        bool use64 = false;
        int32_t first_its = -1;
        int64_t active = read_i64(C, S.nactive);
        while (active > 0 && rep.refinements < MIXED_MAX_ROUNDS && it < opt.max_iters) {
            int32_t its;
            bool hit_cap = false;
            SSP_CUDA(cudaMemsetAsync(Si.nactive, 0, sizeof(int64_t), C.stream));
            if (!use64) {
                k_rhs_masked<float><<<egrid, 256, 0, C.stream>>>(n, ld, r, S.active, r32, R.G);
                SSP_CUDA(cudaMemsetAsync(e32, 0, sizeof(float) * total, C.stream));
                R.run<OP_SQ, float>(r32, nullptr, Si.bnorm2);
                k_cols_init_inner<<<cg, 256, 0, C.stream>>>(ld, k, MIXED_INNER_REDUCTION, S.thr, Si, R.G);
                SSP_CHECK_LAUNCH();
                C.kernels_launched += 2;
                const PcApply pc32f = [&C, &F, V32, n, r32, z32, ld, k, ra](const TrsvShapes* sh, LevelEvents* lev) {
                    return launch_precond<float>(C, F, V32, n, r32, z32, ld, k, ra, sh, lev);
                };
                if (!P32.exec) build_precond_graph(C, F, n, ld, k, sizeof(float), P32, pc32, rep, ra, pc32f);
                int32_t cap = opt.max_iters - it;
                if (first_its >= 0)
                    cap = std::min(cap, std::max(MIXED_MIN_ROUND_ITERS, MIXED_ROUND_ITER_FACTOR * first_its));
                else
                    cap = std::min(cap, std::max(MIXED_MIN_ROUND_ITERS, opt.max_iters / MIXED_FIRST_ROUND_DIV));
                its = pcg_solve<float>(C, n, k, ld, A, aval32, F, pc32f, P32, pc32,
                                       PcgBufs<float>{e32, r32, z32, p32, q32}, Si, R, cap, opt, tm, rep, ra);
                if (first_its < 0) first_its = its;
                hit_cap = its >= cap;
                k_add_into<float><<<grid_for(total, 256, 148 * 16), 256, 0, C.stream>>>(total, e32, x);
            } else {
                if (!e64) e64 = W.get_t<double>("pcgm_e64", total);
                // the FP64 inner solve runs in place on the residual of the active columns and goes straight
                // to (half) the outer threshold
                k_rhs_masked<double><<<egrid, 256, 0, C.stream>>>(n, ld, r, S.active, r, R.G);
                SSP_CUDA(cudaMemsetAsync(e64, 0, sizeof(double) * total, C.stream));
                R.run<OP_SQ, double>(r, nullptr, Si.bnorm2);
                k_cols_init_inner<<<cg, 256, 0, C.stream>>>(ld, k, 0.0, S.thr, Si, R.G);
                SSP_CHECK_LAUNCH();
                C.kernels_launched += 2;
                const PcApply pc64f = [&C, &F, n, r, z, ld, k, ra](const TrsvShapes* sh, LevelEvents* lev) {
                    return launch_precond<double>(C, F, fp64_vals(F), n, r, z, ld, k, ra, sh, lev);
                };
                if (!P64.exec) build_precond_graph(C, F, n, ld, k, sizeof(double), P64, pc64, rep, ra, pc64f);
                its = pcg_solve<double>(C, n, k, ld, A, A.val, F, pc64f, P64, pc64,
                                        PcgBufs<double>{e64, r, z, p, q}, Si, R, opt.max_iters - it, opt, tm, rep,
                                        ra);
                k_add_into<double><<<grid_for(total, 256, 148 * 16), 256, 0, C.stream>>>(total, e64, x);
                rep.fp64_rounds++;
            }
            SSP_CHECK_LAUNCH();
            C.kernels_launched++;
            it += its;
            rep.refinements++;
            // true residual with the FP64 matrix and FP64 x
            ev_resid.begin(C.stream);
            launch_spmm<double>(C, n, A, A.val, x, q, ld, false, k);
            ev_resid.end(C.stream);
            k_true_resid<<<dim3((unsigned)R.nparts, (unsigned)ntiles), RED_THREADS, 0, C.stream>>>(
                n, k, Y, mean, q, r, R.rows_per_blk, ld, R.part, R.G);
            SSP_CHECK_LAUNCH();
            C.kernels_launched += 1 + A.nslabs;
            R.finish(relres);
            SSP_CUDA(cudaMemsetAsync(S.nactive, 0, sizeof(int64_t), C.stream));
            SSP_CUDA(cudaMemsetAsync(worst, 0, sizeof(double), C.stream));
            k_cols_outer<<<cg, 256, 0, C.stream>>>(ns, Si.iters, relres, S, worst);
            SSP_CHECK_LAUNCH();
            C.kernels_launched++;
            active = read_i64(C, S.nactive);
            double hw = 0.0;
            SSP_CUDA(cudaMemcpyAsync(&hw, worst, sizeof(double), cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaStreamSynchronize(C.stream));
            if (opt.verbose)
                fprintf(stderr, "[ssp] refinement %d (%s inner, %d iterations): %lld columns active, worst ratio %.3g\n",
                        rep.refinements, use64 ? "fp64" : "fp32", its, (long long)active, hw);
            if (active > 0 && !use64 && (hw > MIXED_MIN_CONTRACTION || its == 0 || hit_cap)) use64 = true;
        }
    }
    // true relative residual ||(Y - mean) - A x|| / ||Y - mean|| (with the edges' squared diff norms when asked)
    if (lap_eid && d2 && A.nslabs == 1) {
        for (int64_t t = 0; t < ntiles; t++)
            k_spmm_diff<<<dim3(A.grid.x, 1), CH_THREADS, 0, C.stream>>>(
                n, A.chunks[0], A.nchunks[0], A.ptr, A.idx, A.val, lap_eid, x + t * n * TILE, q + t * n * TILE,
                (int32_t)(k - t * TILE), d2, (t == 0 && !d2_accumulate) ? 1 : 0);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += ntiles;
        rep.diff_fused = true;
    } else {
        launch_spmm<double>(C, n, A, A.val, x, q, ld, false, k);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += A.nslabs;
    }
    R.run<OP_SQDIFF_CENTERED, double>(Y, q, relres, mean);
    std::vector<double> hb(ns), hr(ns);
    std::vector<int32_t> hi(ns);
    SSP_CUDA(cudaMemcpyAsync(hb.data(), S.bnorm2, sizeof(double) * ns, cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaMemcpyAsync(hr.data(), relres, sizeof(double) * ns, cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaMemcpyAsync(hi.data(), S.iters, sizeof(int32_t) * ns, cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    double sum_it = 0;
    int64_t cols = 0;
    if (segs) {
        segs->iters.assign(ns, 0);
        segs->relres.assign(ns, 0.0);
    }
    for (int32_t sg = 0; sg < G.nseg; sg++) {
        const int32_t kk = segs ? segs->k[sg] : k;
        for (int32_t j = 0; j < kk; j++) {
            const int64_t o = (int64_t)sg * ld + j;
            double rel = hb[o] > 0 ? sqrt(hr[o]) / sqrt(hb[o]) : 0.0;
            if (h_relres && !segs) h_relres[j] = rel;
            if (h_iters && !segs) h_iters[j] = hi[o];
            if (segs) {
                segs->iters[o] = hi[o];
                segs->relres[o] = rel;
            }
            rep.max_iters_used = std::max(rep.max_iters_used, hi[o]);
            sum_it += hi[o];
            cols++;
            rep.max_relres = std::max(rep.max_relres, rel);
            if (!(rel < 0.01)) rep.not_converged++;
        }
    }
    rep.mean_iters = sum_it / std::max<int64_t>(1, cols);
    rep.ms_spmm = tm.spmm.total_ms();
    rep.n_spmm = (int64_t)tm.spmm.used;
    rep.ms_precond = tm.pc.total_ms();
    rep.n_precond = (int64_t)tm.pc.used;
    rep.ms_loop = tm.loop.total_ms();
    rep.ms_resid = ev_resid.total_ms();
    rep.n_resid = (int64_t)ev_resid.used;
    rep.iters_run = it;
    rep.spmm_slabs = A.nslabs;
    if (x_out) *x_out = x;
}

}  // namespace ssp
