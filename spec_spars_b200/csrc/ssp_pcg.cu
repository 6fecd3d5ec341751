// ssp_pcg.cu -- a8: preconditioned conjugate gradients on all k right-hand sides at once.
//
// Reference: example_pcg_solver (custom_cg.hpp:96-274), called once per sketch column
// (example.cc:552-569).  Per column: b = rhs - mean(rhs) (:132), x0 = 0 (:140), PCG with the
// preconditioner M^{-1} r = L^{-T} D^+ L^{-1} r (:224-235, zero pivots skipped), stop once
// ||r|| <= max(abs_tol, tol ||b||) (the reference's own rule is ||r||^2 <= 2e-7, :159,213), at most
// max_iters iterations (:153), and success iff ||b - A x|| / ||b|| < 0.01 (:251-258).
//
// Layout ("tile-major", tile_off): an n x k block is stored as slabs of n x SSP_TILE doubles.  Every
// kernel works on one tile at a time across all rows, so the rows it gathers (one slab) stay resident
// in L2 while the sparse matrix streams.  Column reductions are two-stage with a fixed order
// (deterministic run to run).
#include "ssp_internal.cuh"

namespace ssp {

constexpr int TILE = SSP_TILE;    // columns per tile
constexpr int SLOTS = 32 / TILE;  // nonzeros processed in parallel per warp
constexpr int ROWS_PER_BLOCK = 8; // warps per 256-thread block, one row each
constexpr int RED_THREADS = 256;  // column reductions: (256 / TILE) row lanes x TILE columns

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

// ---------------------------------------------------------------- column reductions
enum ColOp { OP_SUM = 0, OP_DOT = 1, OP_SQ = 2, OP_SQDIFF_CENTERED = 3 };

// grid (nparts, ntiles); thread = (row lane = tid / 8, column = tid % 8); part[blk][col]
template <int OP>
__global__ void __launch_bounds__(RED_THREADS) k_colred_partial(int64_t n, const double* __restrict__ a,
                                                                const double* __restrict__ b,
                                                                const double* __restrict__ mean, int64_t rows_per_blk,
                                                                int64_t ld, double* __restrict__ part) {
    __shared__ double s[RED_THREADS];
    const int64_t t = blockIdx.y;
    const int c = threadIdx.x % TILE, rl = threadIdx.x / TILE;
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_blk, r1 = min(n, r0 + rows_per_blk);
    const double* at = a + t * n * TILE;
    const double* bt = b ? b + t * n * TILE : nullptr;
    const double mu = (OP == OP_SQDIFF_CENTERED) ? mean[t * TILE + c] : 0.0;
    double acc = 0.0;
    for (int64_t r = r0 + rl; r < r1; r += RED_THREADS / TILE) {
        const double x = at[r * TILE + c];
        if (OP == OP_SUM) acc += x;
        else if (OP == OP_DOT) acc += x * bt[r * TILE + c];
        else if (OP == OP_SQ) acc += x * x;
        else {
            const double d = (x - mu) - bt[r * TILE + c];  // (Y - mean) - A x
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

__global__ void k_colred_final(int64_t ld, int nparts, const double* __restrict__ part, double* __restrict__ out) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ld; c += (int64_t)gridDim.x * blockDim.x) {
        double t = 0.0;
        for (int i = 0; i < nparts; i++) t += part[(int64_t)i * ld + c];
        out[c] = t;
    }
}

struct Reducer {
    Context* C;
    int64_t n, ld;
    int nparts;
    int64_t rows_per_blk;
    double* part;
    void init(Context& c, int64_t n_, int64_t ld_, const char* tag = "pcg_red_part") {
        C = &c;
        n = n_;
        ld = ld_;
        const int64_t ntiles = ld / TILE;
        int64_t target = std::max<int64_t>(8, std::min<int64_t>(1184 / std::max<int64_t>(1, ntiles) + 1, 1024));
        rows_per_blk = std::max<int64_t>(RED_THREADS / TILE, ceil_div<int64_t>(n, target));
        nparts = (int)ceil_div<int64_t>(n, rows_per_blk);
        part = c.ws.get_t<double>(tag, (size_t)nparts * ld);
    }
    template <int OP>
    void run(const double* a, const double* b, double* out, const double* mean = nullptr) {
        dim3 grid((unsigned)nparts, (unsigned)(ld / TILE));
        k_colred_partial<OP><<<grid, RED_THREADS, 0, C->stream>>>(n, a, b, mean, rows_per_blk, ld, part);
        k_colred_final<<<grid_for(ld, 256), 256, 0, C->stream>>>(ld, nparts, part, out);
        SSP_CHECK_LAUNCH();
        C->kernels_launched += 2;
    }
    void finish(double* out) {
        k_colred_final<<<grid_for(ld, 256), 256, 0, C->stream>>>(ld, nparts, part, out);
        SSP_CHECK_LAUNCH();
        C->kernels_launched++;
    }
};

// ---------------------------------------------------------------- elementwise (grid.y = tile)
__global__ void k_center(int64_t n, int32_t k, const double* __restrict__ Y, const double* __restrict__ colsum,
                         double* __restrict__ r, double* __restrict__ x, double* __restrict__ mean) {
    const int64_t t = blockIdx.y;
    const int64_t cnt = n * TILE;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = t * TILE + (i % TILE);
        const int64_t o = t * cnt + i;
        const double mu = c < k ? colsum[c] / (double)n : 0.0;
        if (i < TILE && blockIdx.x == 0) mean[c] = mu;
        r[o] = c < k ? Y[o] - mu : 0.0;
        x[o] = 0.0;
    }
}

// x += alpha p ; r -= alpha q ; partial ||r||^2 per column
__global__ void __launch_bounds__(RED_THREADS) k_axpy_xr_rr(int64_t n, const double* __restrict__ alpha,
                                                            const double* __restrict__ p, const double* __restrict__ q,
                                                            double* __restrict__ x, double* __restrict__ r,
                                                            int64_t rows_per_blk, int64_t ld, double* __restrict__ part) {
    __shared__ double s[RED_THREADS];
    const int64_t t = blockIdx.y;
    const int c = threadIdx.x % TILE, rl = threadIdx.x / TILE;
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_blk, r1 = min(n, r0 + rows_per_blk);
    const double a = alpha[t * TILE + c];
    const int64_t base = t * n * TILE;
    double acc = 0.0;
    for (int64_t row = r0 + rl; row < r1; row += RED_THREADS / TILE) {
        const int64_t o = base + row * TILE + c;
        double rv = r[o];
        if (a != 0.0) {
            x[o] += a * p[o];
            rv -= a * q[o];
            r[o] = rv;
        }
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

__global__ void k_update_p(int64_t n, const double* __restrict__ beta, const double* __restrict__ z,
                           double* __restrict__ p) {
    const int64_t t = blockIdx.y;
    const int64_t cnt = n * TILE;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = t * cnt + i;
        p[o] = z[o] + beta[t * TILE + (i % TILE)] * p[o];
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

__global__ void k_cols_init(int64_t ld, int32_t k, double tol, double abs_tol, ColState S) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ld; c += (int64_t)gridDim.x * blockDim.x) {
        double bn = sqrt(S.bnorm2[c]);
        double thr = tol * bn;
        if (abs_tol > thr) thr = abs_tol;
        S.thr[c] = thr;
        S.rr[c] = S.bnorm2[c];
        int act = (c < k) && (bn > thr);
        S.active[c] = act;
        S.iters[c] = 0;
        S.alpha[c] = 0.0;
        S.beta[c] = 0.0;
        if (act) atomicAdd((unsigned long long*)S.nactive, 1ull);
    }
}

__global__ void k_cols_alpha(int64_t ld, ColState S) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ld; c += (int64_t)gridDim.x * blockDim.x)
        S.alpha[c] = S.active[c] ? S.rz[c] / S.pq[c] : 0.0;
}

__global__ void k_cols_check(int64_t ld, int32_t it, ColState S) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ld; c += (int64_t)gridDim.x * blockDim.x) {
        if (!S.active[c]) continue;
        S.iters[c] = it;
        if (sqrt(S.rr[c]) <= S.thr[c]) S.active[c] = 0;
        else atomicAdd((unsigned long long*)S.nactive, 1ull);
    }
}

__global__ void k_cols_beta(int64_t ld, ColState S) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ld; c += (int64_t)gridDim.x * blockDim.x) {
        double b = 0.0;
        if (S.active[c]) b = S.rz_new[c] / S.rz[c];
        S.beta[c] = b;
        S.rz[c] = S.rz_new[c];
    }
}

// ---------------------------------------------------------------- SpMM and triangular solves
// Warp per row; lane = slot * TILE + column.  xt points at the tile's slab (row stride TILE doubles).
// Two independent gathers per lane per step keep more loads in flight.
__device__ __forceinline__ double warp_row_gather(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                                  const double* __restrict__ val, int64_t row, const double* xt,
                                                  int lane) {
    const int slot = lane / TILE, c = lane % TILE;
    const int64_t e = ptr[row + 1];
    double acc0 = 0.0, acc1 = 0.0;
    int64_t p = ptr[row] + slot;
    for (; p + SLOTS < e; p += 2 * SLOTS) {
        const int32_t i0 = idx[p], i1 = idx[p + SLOTS];
        const double v0 = val[p], v1 = val[p + SLOTS];
        acc0 += v0 * xt[(int64_t)i0 * TILE + c];
        acc1 += v1 * xt[(int64_t)i1 * TILE + c];
    }
    if (p < e) acc0 += val[p] * xt[(int64_t)idx[p] * TILE + c];
    double acc = acc0 + acc1;
#pragma unroll
    for (int o = TILE; o < 32; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

// q = A p for one tile per blockIdx.y; the epilogue accumulates p.q per column into part[blockIdx.x]
__global__ void __launch_bounds__(256) k_spmm_pq(int64_t n, const int64_t* __restrict__ ptr,
                                                 const int32_t* __restrict__ idx, const double* __restrict__ val,
                                                 const double* __restrict__ x, double* __restrict__ y, int64_t ld,
                                                 double* __restrict__ part) {
    __shared__ double s[ROWS_PER_BLOCK][TILE];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t t = blockIdx.y;
    const double* xt = x + t * n * TILE;
    double* yt = y + t * n * TILE;
    const int64_t wstride = (int64_t)gridDim.x * ROWS_PER_BLOCK;
    double dot = 0.0;
    for (int64_t row = (int64_t)blockIdx.x * ROWS_PER_BLOCK + warp; row < n; row += wstride) {
        const double acc = warp_row_gather(ptr, idx, val, row, xt, lane);
        if (lane < TILE) {
            yt[row * TILE + lane] = acc;
            dot += acc * xt[row * TILE + lane];
        }
    }
    if (part) {
        if (lane < TILE) s[warp][lane] = dot;
        __syncthreads();
        if (threadIdx.x < TILE) {
            double tt = s[0][threadIdx.x];
            for (int i = 1; i < ROWS_PER_BLOCK; i++) tt += s[i][threadIdx.x];
            part[(int64_t)blockIdx.x * ld + t * TILE + threadIdx.x] = tt;
        }
    }
}

// forward: y[u] = r[u] - sum_{v<u} L[u,v] y[v]  for the rows of one level
__global__ void __launch_bounds__(256) k_trsv_fwd(int64_t n, const int32_t* __restrict__ rows, int32_t nrows,
                                                  const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                                  const double* __restrict__ val, const double* __restrict__ r,
                                                  double* y) {
    const int lane = threadIdx.x & 31;
    const int64_t toff = (int64_t)blockIdx.y * n * TILE;
    const int wstride = gridDim.x * ROWS_PER_BLOCK;
    for (int i = blockIdx.x * ROWS_PER_BLOCK + (threadIdx.x >> 5); i < nrows; i += wstride) {
        const int64_t u = rows[i];
        const double acc = warp_row_gather(ptr, idx, val, u, y + toff, lane);
        if (lane < TILE) {
            const int64_t o = toff + u * TILE + lane;
            y[o] = r[o] - acc;
        }
    }
}

// backward (in place over y): z[u] = y[u]/D[u] - sum_{v>u} L[v,u] z[v]
__global__ void __launch_bounds__(256) k_trsv_bwd(int64_t n, const int32_t* __restrict__ rows, int32_t nrows,
                                                  const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                                  const double* __restrict__ val, const double* __restrict__ D,
                                                  double* yz) {
    const int lane = threadIdx.x & 31;
    const int64_t toff = (int64_t)blockIdx.y * n * TILE;
    const int wstride = gridDim.x * ROWS_PER_BLOCK;
    for (int i = blockIdx.x * ROWS_PER_BLOCK + (threadIdx.x >> 5); i < nrows; i += wstride) {
        const int64_t u = rows[i];
        const double acc = warp_row_gather(ptr, idx, val, u, yz + toff, lane);
        if (lane < TILE) {
            const int64_t o = toff + u * TILE + lane;
            const double d = D[u];
            const double yu = yz[o];
            yz[o] = (d != 0.0 ? yu / d : yu) - acc;
        }
    }
}


// ---------------------------------------------------------------- chunked gather (SpMM-shaped work)
// A chunk is a run of consecutive stored rows with at most CHUNK_CAP entries and CHUNK_ROWS rows (or
// one longer row).  Each warp owns whole chunks: it stages the chunk's (index, value) pairs in its own
// shared-memory slice with coalesced streaming loads (the matrix is read once per tile and should not
// evict the gathered slab from L2), then every (row, column) lane pair sums its row with independent
// gathers from the tile slab.  Warps never wait for each other.  Modes: SpMM (+ p.q partials),
// forward solve, backward solve.
enum { M_SPMM = 0, M_FWD = 1, M_BWD = 2 };
constexpr int CH_THREADS = 256;
constexpr int CH_WARPS = CH_THREADS / 32;

template <int MODE>
__device__ __forceinline__ void chunk_epilogue(double* out, const double* aux, const double* xt, int64_t toff,
                                               int64_t v, int col, double acc, double& dot) {
    const int64_t o = toff + v * TILE + col;
    if (MODE == M_SPMM) {
        out[o] = acc;
        dot += acc * xt[v * TILE + col];
    } else if (MODE == M_FWD) {
        out[o] = aux[o] - acc;
    } else {
        const double d = aux[v];
        const double yu = out[o];
        out[o] = (d != 0.0 ? yu / d : yu) - acc;
    }
}

template <int MODE>
__global__ void __launch_bounds__(CH_THREADS) k_chunked(int64_t n, const int32_t* __restrict__ cstart, int32_t nchunks,
                                                        const int64_t* __restrict__ ptr,
                                                        const int32_t* __restrict__ idx,
                                                        const double* __restrict__ val,
                                                        const int32_t* __restrict__ rowmap, const double* xsrc,
                                                        double* out, const double* __restrict__ aux, int64_t ld,
                                                        double* __restrict__ part) {
    __shared__ int32_t s_idx[CH_WARPS][CHUNK_CAP];
    __shared__ double s_val[CH_WARPS][CHUNK_CAP];
    __shared__ int32_t s_ptr[CH_WARPS][CHUNK_ROWS + 1];
    __shared__ double s_red[CH_THREADS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t t = blockIdx.y;
    const int64_t toff = t * n * TILE;
    const double* xt = xsrc + toff;
    int32_t* si = s_idx[w];
    double* sv = s_val[w];
    int32_t* sp = s_ptr[w];
    double dot = 0.0;  // SpMM: per-lane partial of p.q for column (lane % TILE)
    for (int32_t c = blockIdx.x * CH_WARPS + w; c < nchunks; c += gridDim.x * CH_WARPS) {
        const int32_t r0 = cstart[c], r1 = cstart[c + 1];
        const int64_t e0 = ptr[r0], e1 = ptr[r1];
        const int64_t ne = e1 - e0;
        if (ne <= CHUNK_CAP) {
            for (int64_t i = lane; i < ne; i += 32) {
                si[i] = __ldcs(idx + e0 + i);
                sv[i] = __ldcs(val + e0 + i);
            }
            for (int32_t i = lane; i <= r1 - r0; i += 32) sp[i] = (int32_t)(ptr[r0 + i] - e0);
            __syncwarp();
            const int32_t pairs = (r1 - r0) * TILE;
            for (int32_t pr = lane; pr < pairs; pr += 32) {
                const int32_t rr = pr / TILE, col = pr % TILE;
                const int32_t q0 = sp[rr], q1 = sp[rr + 1];
                double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
                int32_t q = q0;
                for (; q + 3 < q1; q += 4) {
                    a0 += sv[q] * xt[(int64_t)si[q] * TILE + col];
                    a1 += sv[q + 1] * xt[(int64_t)si[q + 1] * TILE + col];
                    a2 += sv[q + 2] * xt[(int64_t)si[q + 2] * TILE + col];
                    a3 += sv[q + 3] * xt[(int64_t)si[q + 3] * TILE + col];
                }
                for (; q < q1; q++) a0 += sv[q] * xt[(int64_t)si[q] * TILE + col];
                const int64_t row = r0 + rr;
                chunk_epilogue<MODE>(out, aux, xt, toff, rowmap ? rowmap[row] : row, col, (a0 + a1) + (a2 + a3), dot);
            }
            __syncwarp();
        } else {
            // one long row: (32 / TILE) entry slots x TILE columns per step, then a reduction over the slots
            const int slot = lane / TILE, col = lane % TILE;
            double a0 = 0.0, a1 = 0.0;
            int64_t q = e0 + slot;
            for (; q + SLOTS < e1; q += 2 * SLOTS) {
                a0 += __ldcs(val + q) * xt[(int64_t)__ldcs(idx + q) * TILE + col];
                a1 += __ldcs(val + q + SLOTS) * xt[(int64_t)__ldcs(idx + q + SLOTS) * TILE + col];
            }
            if (q < e1) a0 += __ldcs(val + q) * xt[(int64_t)__ldcs(idx + q) * TILE + col];
            double acc = a0 + a1;
#pragma unroll
            for (int o = TILE; o < 32; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane < TILE) chunk_epilogue<MODE>(out, aux, xt, toff, rowmap ? rowmap[r0] : r0, col, acc, dot);
        }
    }
    if (MODE == M_SPMM && part) {
        s_red[threadIdx.x] = dot;
        __syncthreads();
        if (threadIdx.x < TILE) {
            double tt = 0.0;
            for (int i = 0; i < CH_THREADS / TILE; i++) tt += s_red[i * TILE + threadIdx.x];
            part[(int64_t)blockIdx.x * ld + t * TILE + threadIdx.x] = tt;
        }
    }
}

// blocks per tile: about one wave of resident blocks, so the gathered slab of the tile being worked
// on is the only one live in L2
static int chunk_blocks(int32_t nchunks) {
    return std::max(1, std::min((nchunks + CH_WARPS - 1) / CH_WARPS, 148 * 6));
}

// Runs of thin levels: the k columns are independent, so one block per 8-column tile can walk a run
// of consecutive levels on its own, with only a block barrier between levels (its own writes are the
// only values it reads back).  y is read and written in place: no read-only cache path.
constexpr int RUN_THREADS = 512;
constexpr int THIN_ROWS = 64;

// rows[i] is the vertex of stored row i; ptr/idx/val are in storage order
__global__ void __launch_bounds__(RUN_THREADS) k_trsv_fwd_run(int64_t n, const int32_t* __restrict__ rows,
                                                              const int32_t* __restrict__ lptr, int32_t l0,
                                                              int32_t l1, const int64_t* __restrict__ ptr,
                                                              const int32_t* __restrict__ idx,
                                                              const double* __restrict__ val,
                                                              const double* __restrict__ r, double* y) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = RUN_THREADS / 32;
    const int64_t toff = (int64_t)blockIdx.x * n * TILE;
    for (int32_t l = l0; l < l1; l++) {
        const int32_t s = lptr[l], e = lptr[l + 1];
        for (int32_t i = s + warp; i < e; i += nwarp) {
            const int64_t u = rows[i];
            const double acc = warp_row_gather(ptr, idx, val, i, y + toff, lane);
            if (lane < TILE) {
                const int64_t o = toff + u * TILE + lane;
                y[o] = r[o] - acc;
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(RUN_THREADS) k_trsv_bwd_run(int64_t n, const int32_t* __restrict__ rows,
                                                              const int32_t* __restrict__ lptr, int32_t l0,
                                                              int32_t l1, const int64_t* __restrict__ ptr,
                                                              const int32_t* __restrict__ idx,
                                                              const double* __restrict__ val,
                                                              const double* __restrict__ D, double* yz) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = RUN_THREADS / 32;
    const int64_t toff = (int64_t)blockIdx.x * n * TILE;
    for (int32_t l = l1 - 1; l >= l0; l--) {
        const int32_t s = lptr[l], e = lptr[l + 1];
        for (int32_t i = s + warp; i < e; i += nwarp) {
            const int64_t u = rows[i];
            const double acc = warp_row_gather(ptr, idx, val, i, yz + toff, lane);
            if (lane < TILE) {
                const int64_t o = toff + u * TILE + lane;
                const double d = D[u];
                const double yu = yz[o];
                yz[o] = (d != 0.0 ? yu / d : yu) - acc;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- preconditioner as a CUDA graph
struct Precond {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~Precond() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

// level schedule: maximal runs of thin levels become one launch; wide levels launch on their own
static std::vector<std::pair<int32_t, int32_t>> level_segments(const DevFactor& F) {
    std::vector<std::pair<int32_t, int32_t>> seg;
    int32_t l = 0;
    while (l < F.num_levels) {
        int32_t r = l;
        while (r < F.num_levels && F.level_ptr[r + 1] - F.level_ptr[r] <= THIN_ROWS) r++;
        if (r - l >= 2) {
            seg.push_back({l, r});  // run [l, r)
            l = r;
        } else {
            seg.push_back({l, l + 1});
            l++;
        }
    }
    return seg;
}

static int64_t launch_precond(Context& C, const DevFactor& F, int64_t n, const double* r, double* y, int64_t ld) {
    const int ntiles = (int)(ld / TILE);
    int64_t launches = 0;
    const auto seg = level_segments(F);
    for (size_t i = 0; i < seg.size(); i++) {
        const int32_t l0 = seg[i].first, l1 = seg[i].second;
        if (l1 - l0 >= 2) {
            k_trsv_fwd_run<<<ntiles, RUN_THREADS, 0, C.stream>>>(n, F.level_rows, F.level_ptr_d, l0, l1, F.prow_ptr,
                                                                  F.prow_idx, F.prow_val, r, y);
        } else {
            const int32_t c0 = F.fchunk_lvl[l0], nc = F.fchunk_lvl[l0 + 1] - c0;
            if (nc == 0) continue;
            dim3 grid((unsigned)chunk_blocks(nc), (unsigned)ntiles);
            k_chunked<M_FWD><<<grid, CH_THREADS, 0, C.stream>>>(n, F.fchunk + c0, nc, F.prow_ptr, F.prow_idx,
                                                                 F.prow_val, F.level_rows, y, y, r, ld, nullptr);
        }
        launches++;
    }
    for (size_t i = seg.size(); i-- > 0;) {
        const int32_t l0 = seg[i].first, l1 = seg[i].second;
        if (l1 - l0 >= 2) {
            k_trsv_bwd_run<<<ntiles, RUN_THREADS, 0, C.stream>>>(n, F.level_rows, F.level_ptr_d, l0, l1, F.pcol_ptr,
                                                                  F.pcol_idx, F.pcol_val, F.D, y);
        } else {
            const int32_t c0 = F.bchunk_lvl[l0], nc = F.bchunk_lvl[l0 + 1] - c0;
            if (nc == 0) continue;
            dim3 grid((unsigned)chunk_blocks(nc), (unsigned)ntiles);
            k_chunked<M_BWD><<<grid, CH_THREADS, 0, C.stream>>>(n, F.bchunk + c0, nc, F.pcol_ptr, F.pcol_idx,
                                                                 F.pcol_val, F.level_rows, y, y, F.D, ld, nullptr);
        }
        launches++;
    }
    SSP_CHECK_LAUNCH();
    return launches;
}

static void build_precond_graph(Context& C, const DevFactor& F, int64_t n, const double* r, double* y, int64_t ld,
                                Precond& P, int64_t& launches) {
    SSP_CUDA(cudaStreamBeginCapture(C.stream, cudaStreamCaptureModeThreadLocal));
    try {
        launches = launch_precond(C, F, n, r, y, ld);
    } catch (...) {
        cudaGraph_t g;
        cudaStreamEndCapture(C.stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    SSP_CUDA(cudaStreamEndCapture(C.stream, &P.graph));
    SSP_CUDA(cudaGraphInstantiate(&P.exec, P.graph, 0));
}

// apply M^{-1} to R into Z once (tile-major n x ld blocks; stage entry point)
void precond_apply_device(Context& C, const DevFactor& F, const double* R, double* Z, int64_t ld) {
    int64_t l = launch_precond(C, F, F.n, R, Z, ld);
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

// ---------------------------------------------------------------- driver
// Y: tile-major n x ld (ld = round8(k)), read only.  The solution stays in the workspace buffer
// "pcg_x" (tile-major); *x_out points at it.
void pcg_device(Context& C, int64_t n, const int64_t* lap_ptr, const int32_t* lap_idx, const double* lap_val,
                const DevFactor& F, const double* Y, int32_t k, const double** x_out, const PcgOptions& opt,
                PcgReport& rep, int32_t* h_iters, double* h_relres) {
    SSP_REQUIRE(k > 0, SSP_ERR_INVALID, "pcg: k must be positive");
    const int64_t ld = ((int64_t)k + TILE - 1) / TILE * TILE;
    const int64_t ntiles = ld / TILE;
    const int64_t total = n * ld;
    Workspace& W = C.ws;
    double* x = W.get_t<double>("pcg_x", total);
    double* r = W.get_t<double>("pcg_r", total);
    double* z = W.get_t<double>("pcg_z", total);
    double* p = W.get_t<double>("pcg_p", total);
    double* q = W.get_t<double>("pcg_q", total);
    double* colv = W.get_t<double>("pcg_cols", 11 * ld);
    int32_t* coli = W.get_t<int32_t>("pcg_coli", 2 * ld);
    int64_t* nact = W.get_t<int64_t>("pcg_nactive", 1);
    ColState S{colv, colv + ld, colv + 2 * ld, colv + 3 * ld, colv + 4 * ld, colv + 5 * ld, colv + 6 * ld,
               colv + 7 * ld, coli, coli + ld, nact};
    double* colsum = colv + 8 * ld;
    double* relres = colv + 9 * ld;
    double* mean = colv + 10 * ld;
    Reducer R;
    R.init(C, n, ld);
    // SpMM: row-aligned chunks of the Laplacian, about one wave of blocks per tile
    std::vector<int32_t> achunks;
    {
        std::vector<int64_t> hp(n + 1);
        SSP_CUDA(cudaMemcpyAsync(hp.data(), lap_ptr, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
        make_chunks(hp, 0, (int32_t)n, achunks);
        achunks.push_back((int32_t)n);
    }
    const int32_t anch = (int32_t)achunks.size() - 1;
    int32_t* d_achunks = W.get_t<int32_t>("pcg_achunks", achunks.size());
    SSP_CUDA(cudaMemcpyAsync(d_achunks, achunks.data(), sizeof(int32_t) * achunks.size(), cudaMemcpyHostToDevice,
                             C.stream));
    const int spmm_bx = chunk_blocks(anch);
    double* spmm_part = W.get_t<double>("pcg_spmm_part", (size_t)spmm_bx * ld);
    const dim3 sgrid((unsigned)spmm_bx, (unsigned)ntiles);
    const dim3 egrid((unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div<int64_t>(n * TILE, 256),
                                                                      2048 / std::max<int64_t>(1, ntiles) + 4)),
                     (unsigned)ntiles);
    const int cg = grid_for(ld, 256);

    // r = Y - mean(Y); x = 0; ||b||^2
    R.run<OP_SUM>(Y, nullptr, colsum);
    k_center<<<egrid, 256, 0, C.stream>>>(n, k, Y, colsum, r, x, mean);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    R.run<OP_SQ>(r, nullptr, S.bnorm2);
    SSP_CUDA(cudaMemsetAsync(nact, 0, sizeof(int64_t), C.stream));
    k_cols_init<<<cg, 256, 0, C.stream>>>(ld, k, opt.tol, opt.abs_tol, S);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    int64_t active = read_i64(C, nact);

    Precond P;
    int64_t pc_launches = 0;
    int32_t it = 0;
    EventPairs ev_spmm, ev_pc, ev_loop;
    if (active > 0) {
        build_precond_graph(C, F, n, r, z, ld, P, pc_launches);
        ev_pc.begin(C.stream);
        SSP_CUDA(cudaGraphLaunch(P.exec, C.stream));
        ev_pc.end(C.stream);
        C.kernels_launched += pc_launches;
        R.run<OP_DOT>(r, z, S.rz);
        SSP_CUDA(cudaMemcpyAsync(p, z, sizeof(double) * total, cudaMemcpyDeviceToDevice, C.stream));
        ev_loop.begin(C.stream);
        while (it < opt.max_iters) {
            ev_spmm.begin(C.stream);
            k_chunked<M_SPMM><<<sgrid, CH_THREADS, 0, C.stream>>>(n, d_achunks, anch, lap_ptr, lap_idx, lap_val,
                                                                   nullptr, p, q, nullptr, ld, spmm_part);
            ev_spmm.end(C.stream);
            k_colred_final<<<cg, 256, 0, C.stream>>>(ld, spmm_bx, spmm_part, S.pq);
            k_cols_alpha<<<cg, 256, 0, C.stream>>>(ld, S);
            k_axpy_xr_rr<<<dim3((unsigned)R.nparts, (unsigned)ntiles), RED_THREADS, 0, C.stream>>>(
                n, S.alpha, p, q, x, r, R.rows_per_blk, ld, R.part);
            SSP_CHECK_LAUNCH();
            C.kernels_launched += 4;
            R.finish(S.rr);
            it++;
            SSP_CUDA(cudaMemsetAsync(nact, 0, sizeof(int64_t), C.stream));
            k_cols_check<<<cg, 256, 0, C.stream>>>(ld, it, S);
            SSP_CHECK_LAUNCH();
            C.kernels_launched++;
            active = read_i64(C, nact);
            if (opt.history) {
                std::vector<double> hrr(k), hbb(k);
                SSP_CUDA(cudaMemcpyAsync(hrr.data(), S.rr, sizeof(double) * k, cudaMemcpyDeviceToHost, C.stream));
                SSP_CUDA(cudaMemcpyAsync(hbb.data(), S.bnorm2, sizeof(double) * k, cudaMemcpyDeviceToHost, C.stream));
                SSP_CUDA(cudaStreamSynchronize(C.stream));
                double mx = 0.0;
                for (int32_t j = 0; j < k; j++)
                    if (hbb[j] > 0) mx = std::max(mx, std::sqrt(hrr[j] / hbb[j]));
                opt.history->push_back(mx);
            }
            if (opt.verbose && (it % 10 == 0 || active == 0))
                fprintf(stderr, "[ssp] pcg iter %d: %lld columns active\n", it, (long long)active);
            if (active == 0) break;
            ev_pc.begin(C.stream);
            SSP_CUDA(cudaGraphLaunch(P.exec, C.stream));
            ev_pc.end(C.stream);
            C.kernels_launched += pc_launches;
            R.run<OP_DOT>(r, z, S.rz_new);
            k_cols_beta<<<cg, 256, 0, C.stream>>>(ld, S);
            k_update_p<<<egrid, 256, 0, C.stream>>>(n, S.beta, z, p);
            SSP_CHECK_LAUNCH();
            C.kernels_launched += 2;
        }
        ev_loop.end(C.stream);
    }
    // true relative residual ||(Y - mean) - A x|| / ||Y - mean||
    k_chunked<M_SPMM><<<sgrid, CH_THREADS, 0, C.stream>>>(n, d_achunks, anch, lap_ptr, lap_idx, lap_val, nullptr, x,
                                                           q, nullptr, ld, nullptr);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    R.run<OP_SQDIFF_CENTERED>(Y, q, relres, mean);
    std::vector<double> hb(ld), hr(ld);
    std::vector<int32_t> hi(ld);
    SSP_CUDA(cudaMemcpyAsync(hb.data(), S.bnorm2, sizeof(double) * ld, cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaMemcpyAsync(hr.data(), relres, sizeof(double) * ld, cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaMemcpyAsync(hi.data(), S.iters, sizeof(int32_t) * ld, cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    rep = PcgReport();
    double sum_it = 0;
    for (int32_t j = 0; j < k; j++) {
        double rel = hb[j] > 0 ? sqrt(hr[j]) / sqrt(hb[j]) : 0.0;
        if (h_relres) h_relres[j] = rel;
        if (h_iters) h_iters[j] = hi[j];
        rep.max_iters_used = std::max(rep.max_iters_used, hi[j]);
        sum_it += hi[j];
        rep.max_relres = std::max(rep.max_relres, rel);
        if (!(rel < 0.01)) rep.not_converged++;
    }
    rep.mean_iters = sum_it / k;
    rep.ms_spmm = ev_spmm.total_ms();
    rep.n_spmm = (int64_t)ev_spmm.used;
    rep.ms_precond = ev_pc.total_ms();
    rep.n_precond = (int64_t)ev_pc.used;
    rep.ms_loop = ev_loop.total_ms();
    rep.iters_run = it;
    if (x_out) *x_out = x;
}

}  // namespace ssp
