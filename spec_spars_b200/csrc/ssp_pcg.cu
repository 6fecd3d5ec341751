// ssp_pcg.cu -- a8: preconditioned conjugate gradients on all k right-hand sides at once.
//
// Reference: example_pcg_solver (custom_cg.hpp:96-274), called once per sketch column
// (example.cc:552-569).  Per column: b = rhs - mean(rhs) (:132), x0 = 0 (:140), PCG with the
// preconditioner M^{-1} r = L^{-T} D^+ L^{-1} r (:224-235, zero pivots skipped), stop once
// ||r|| <= max(abs_tol, tol ||b||) (the reference's own rule is ||r||^2 <= 2e-7, :159,213), at most
// max_iters iterations (:153), and success iff ||b - A x|| / ||b|| < 0.01 (:251-258).
//
// Layout: every n x k block is row-major with a leading dimension ld (a multiple of 8).  Work is
// split into 8-column tiles (64 bytes per row): one launch walks the rows of one tile while
// neighbouring blocks work on the same tile, so the gathered rows of that tile (n*64 bytes)
// stay in L2.  Reductions are per column, two-stage, in a fixed order (deterministic).
#include "ssp_internal.cuh"

namespace ssp {

constexpr int TILE = 8;          // columns per tile
constexpr int SLOTS = 32 / TILE; // nonzeros processed in parallel per warp
constexpr int ROWS_PER_BLOCK = 8;

// ---------------------------------------------------------------- column reductions
enum ColOp { OP_SUM = 0, OP_DOT = 1, OP_SQ = 2, OP_SQDIFF = 3 };

constexpr int RED_ROWS = 8;   // threadIdx.y
constexpr int RED_COLS = 32;  // threadIdx.x

template <int OP>
__global__ void k_colred_partial(int64_t n, int64_t ld, const double* __restrict__ a, const double* __restrict__ b,
                                 int64_t rows_per_blk, double* __restrict__ part) {
    __shared__ double s[RED_ROWS][RED_COLS];
    const int64_t col = (int64_t)blockIdx.y * RED_COLS + threadIdx.x;
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_blk;
    const int64_t r1 = min(n, r0 + rows_per_blk);
    double acc = 0.0;
    if (col < ld) {
        for (int64_t r = r0 + threadIdx.y; r < r1; r += RED_ROWS) {
            double x = a[r * ld + col];
            if (OP == OP_SUM) acc += x;
            else if (OP == OP_DOT) acc += x * b[r * ld + col];
            else if (OP == OP_SQ) acc += x * x;
            else {
                double d = x - b[r * ld + col];
                acc += d * d;
            }
        }
    }
    s[threadIdx.y][threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.y == 0 && col < ld) {
        double t = s[0][threadIdx.x];
        for (int i = 1; i < RED_ROWS; i++) t += s[i][threadIdx.x];
        part[(int64_t)blockIdx.x * ld + col] = t;
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
    void init(Context& c, int64_t n_, int64_t ld_) {
        C = &c;
        n = n_;
        ld = ld_;
        int64_t target = std::max<int64_t>(1, std::min<int64_t>(592 / std::max<int64_t>(1, ceil_div<int64_t>(ld, 32)), 4096));
        target = std::max<int64_t>(target, 8);
        rows_per_blk = std::max<int64_t>(RED_ROWS, ceil_div<int64_t>(n, target));
        nparts = (int)ceil_div<int64_t>(n, rows_per_blk);
        part = c.ws.get_t<double>("pcg_red_part", (size_t)nparts * ld);
    }
    template <int OP>
    void run(const double* a, const double* b, double* out) {
        dim3 grid((unsigned)nparts, (unsigned)ceil_div<int64_t>(ld, RED_COLS));
        dim3 block(RED_COLS, RED_ROWS);
        k_colred_partial<OP><<<grid, block, 0, C->stream>>>(n, ld, a, b, rows_per_blk, part);
        k_colred_final<<<grid_for(ld, 256), 256, 0, C->stream>>>(ld, nparts, part, out);
        SSP_CHECK_LAUNCH();
        C->kernels_launched += 2;
    }
};

// ---------------------------------------------------------------- elementwise
__global__ void k_center(int64_t n, int64_t ld, int32_t k, const double* __restrict__ Y, int64_t ldy,
                         const double* __restrict__ colsum, double* __restrict__ b, double* __restrict__ r,
                         double* __restrict__ x) {
    const int64_t total = n * ld;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t row = i / ld, col = i - row * ld;
        double v = 0.0;
        if (col < k) v = Y[row * ldy + col] - colsum[col] / (double)n;
        b[i] = v;
        r[i] = v;
        x[i] = 0.0;
    }
}

__global__ void k_axpy_xr(int64_t total, int64_t ld, const double* __restrict__ alpha, const double* __restrict__ p,
                          const double* __restrict__ q, double* __restrict__ x, double* __restrict__ r) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        double a = alpha[i % ld];
        if (a != 0.0) {
            x[i] += a * p[i];
            r[i] -= a * q[i];
        }
    }
}

__global__ void k_update_p(int64_t total, int64_t ld, const double* __restrict__ beta, const double* __restrict__ z,
                           double* __restrict__ p) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + beta[i % ld] * p[i];
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
// Warp per row; lane = slot * TILE + column.  Row entries are visited in stored order by slot,
// partial sums are combined across slots with shuffles.
__device__ __forceinline__ double warp_row_gather(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                                  const double* __restrict__ val, int64_t row,
                                                  const double* __restrict__ x, int64_t ld, int64_t colbase,
                                                  int lane) {
    const int slot = lane / TILE, c = lane % TILE;
    double acc = 0.0;
    for (int64_t p = ptr[row] + slot; p < ptr[row + 1]; p += SLOTS) acc += val[p] * x[(int64_t)idx[p] * ld + colbase + c];
#pragma unroll
    for (int o = TILE; o < 32; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

__global__ void __launch_bounds__(256) k_spmm(int64_t n, const int64_t* __restrict__ ptr,
                                              const int32_t* __restrict__ idx, const double* __restrict__ val,
                                              const double* __restrict__ x, double* __restrict__ y, int64_t ld) {
    const int lane = threadIdx.x & 31;
    const int64_t colbase = (int64_t)blockIdx.y * TILE;
    const int64_t wstride = (int64_t)gridDim.x * ROWS_PER_BLOCK;
    for (int64_t row = (int64_t)blockIdx.x * ROWS_PER_BLOCK + (threadIdx.x >> 5); row < n; row += wstride) {
        double acc = warp_row_gather(ptr, idx, val, row, x, ld, colbase, lane);
        if (lane < TILE) y[row * ld + colbase + lane] = acc;
    }
}

// forward: y[u] = r[u] - sum_{v<u} L[u,v] y[v]  for the rows of one level
__global__ void __launch_bounds__(256) k_trsv_fwd(const int32_t* __restrict__ rows, int32_t nrows,
                                                  const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                                  const double* __restrict__ val, const double* __restrict__ r,
                                                  double* __restrict__ y, int64_t ld) {
    const int lane = threadIdx.x & 31;
    const int64_t colbase = (int64_t)blockIdx.y * TILE;
    const int wstride = gridDim.x * ROWS_PER_BLOCK;
    for (int i = blockIdx.x * ROWS_PER_BLOCK + (threadIdx.x >> 5); i < nrows; i += wstride) {
        const int64_t u = rows[i];
        double acc = warp_row_gather(ptr, idx, val, u, y, ld, colbase, lane);
        if (lane < TILE) {
            const int64_t o = u * ld + colbase + lane;
            y[o] = r[o] - acc;
        }
    }
}

// backward (in place over y): z[u] = y[u]/D[u] - sum_{v>u} L[v,u] z[v]
__global__ void __launch_bounds__(256) k_trsv_bwd(const int32_t* __restrict__ rows, int32_t nrows,
                                                  const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                                  const double* __restrict__ val, const double* __restrict__ D,
                                                  double* __restrict__ yz, int64_t ld) {
    const int lane = threadIdx.x & 31;
    const int64_t colbase = (int64_t)blockIdx.y * TILE;
    const int wstride = gridDim.x * ROWS_PER_BLOCK;
    for (int i = blockIdx.x * ROWS_PER_BLOCK + (threadIdx.x >> 5); i < nrows; i += wstride) {
        const int64_t u = rows[i];
        double acc = warp_row_gather(ptr, idx, val, u, yz, ld, colbase, lane);
        if (lane < TILE) {
            const int64_t o = u * ld + colbase + lane;
            const double d = D[u];
            const double yu = yz[o];
            yz[o] = (d != 0.0 ? yu / d : yu) - acc;
        }
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

static int64_t launch_precond(Context& C, const DevFactor& F, const double* r, double* y, int64_t ld) {
    const int ntiles = (int)(ld / TILE);
    int64_t launches = 0;
    for (int32_t l = 0; l < F.num_levels; l++) {
        const int32_t s = F.level_ptr[l], c = F.level_ptr[l + 1] - s;
        if (c == 0) continue;
        dim3 grid((unsigned)std::min<int64_t>(ceil_div<int64_t>(c, ROWS_PER_BLOCK), 592), (unsigned)ntiles);
        k_trsv_fwd<<<grid, 256, 0, C.stream>>>(F.level_rows + s, c, F.row_ptr, F.row_idx, F.row_val, r, y, ld);
        launches++;
    }
    for (int32_t l = F.num_levels - 1; l >= 0; l--) {
        const int32_t s = F.level_ptr[l], c = F.level_ptr[l + 1] - s;
        if (c == 0) continue;
        dim3 grid((unsigned)std::min<int64_t>(ceil_div<int64_t>(c, ROWS_PER_BLOCK), 592), (unsigned)ntiles);
        k_trsv_bwd<<<grid, 256, 0, C.stream>>>(F.level_rows + s, c, F.col_ptr, F.col_idx, F.col_val, F.D, y, ld);
        launches++;
    }
    SSP_CHECK_LAUNCH();
    return launches;
}

static void build_precond_graph(Context& C, const DevFactor& F, const double* r, double* y, int64_t ld, Precond& P,
                                int64_t& launches) {
    SSP_CUDA(cudaStreamBeginCapture(C.stream, cudaStreamCaptureModeThreadLocal));
    try {
        launches = launch_precond(C, F, r, y, ld);
    } catch (...) {
        cudaGraph_t g;
        cudaStreamEndCapture(C.stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    SSP_CUDA(cudaStreamEndCapture(C.stream, &P.graph));
    SSP_CUDA(cudaGraphInstantiate(&P.exec, P.graph, 0));
}

// apply M^{-1} to R (n x ld) into Z (n x ld) once (stage entry point)
void precond_apply_device(Context& C, const DevFactor& F, const double* R, double* Z, int64_t ld) {
    int64_t l = launch_precond(C, F, R, Z, ld);
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
void pcg_device(Context& C, int64_t n, const int64_t* lap_ptr, const int32_t* lap_idx, const double* lap_val,
                const DevFactor& F, const double* Y, int32_t k, int64_t ldy, double* Zout, const PcgOptions& opt,
                PcgReport& rep, int32_t* h_iters, double* h_relres) {
    SSP_REQUIRE(k > 0, SSP_ERR_INVALID, "pcg: k must be positive");
    const int64_t ld = ((int64_t)k + TILE - 1) / TILE * TILE;
    const int64_t total = n * ld;
    Workspace& W = C.ws;
    double* b = W.get_t<double>("pcg_b", total);
    double* x = W.get_t<double>("pcg_x", total);
    double* r = W.get_t<double>("pcg_r", total);
    double* z = W.get_t<double>("pcg_z", total);
    double* p = W.get_t<double>("pcg_p", total);
    double* q = W.get_t<double>("pcg_q", total);
    double* colv = W.get_t<double>("pcg_cols", 10 * ld);
    int32_t* coli = W.get_t<int32_t>("pcg_coli", 2 * ld);
    int64_t* nact = W.get_t<int64_t>("pcg_nactive", 1);
    ColState S{colv, colv + ld, colv + 2 * ld, colv + 3 * ld, colv + 4 * ld, colv + 5 * ld, colv + 6 * ld,
               colv + 7 * ld, coli, coli + ld, nact};
    double* colsum = colv + 8 * ld;
    double* relres = colv + 9 * ld;
    Reducer R;
    R.init(C, n, ld);
    const int eg = grid_for(total, 256, 148 * 16);
    const int cg = grid_for(ld, 256);
    const dim3 sgrid((unsigned)std::min<int64_t>(ceil_div<int64_t>(n, ROWS_PER_BLOCK), 592), (unsigned)(ld / TILE));

    // b = Y - mean(Y); x = 0; r = b  (Y may have ld != ldy; colsum over the first k columns)
    {
        // column sums of Y with its own leading dimension
        Reducer RY;
        RY.C = &C;
        RY.n = n;
        RY.ld = ldy;
        RY.rows_per_blk = R.rows_per_blk;
        RY.nparts = R.nparts;
        RY.part = W.get_t<double>("pcg_red_party", (size_t)RY.nparts * ldy);
        double* ysum = W.get_t<double>("pcg_ysum", ldy);
        RY.run<OP_SUM>(Y, nullptr, ysum);
        k_center<<<eg, 256, 0, C.stream>>>(n, ld, k, Y, ldy, ysum, b, r, x);
        SSP_CHECK_LAUNCH();
        C.kernels_launched++;
    }
    R.run<OP_SQ>(b, nullptr, S.bnorm2);
    SSP_CUDA(cudaMemsetAsync(nact, 0, sizeof(int64_t), C.stream));
    k_cols_init<<<cg, 256, 0, C.stream>>>(ld, k, opt.tol, opt.abs_tol, S);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    int64_t active = read_i64(C, nact);

    Precond P;
    int64_t pc_launches = 0;
    int32_t it = 0;
    EventPairs ev_spmm, ev_pc;
    if (active > 0) {
        build_precond_graph(C, F, r, z, ld, P, pc_launches);
        ev_pc.begin(C.stream);
        SSP_CUDA(cudaGraphLaunch(P.exec, C.stream));
        ev_pc.end(C.stream);
        C.kernels_launched += pc_launches;
        R.run<OP_DOT>(r, z, S.rz);
        SSP_CUDA(cudaMemcpyAsync(p, z, sizeof(double) * total, cudaMemcpyDeviceToDevice, C.stream));
        while (it < opt.max_iters) {
            ev_spmm.begin(C.stream);
            k_spmm<<<sgrid, 256, 0, C.stream>>>(n, lap_ptr, lap_idx, lap_val, p, q, ld);
            ev_spmm.end(C.stream);
            SSP_CHECK_LAUNCH();
            C.kernels_launched++;
            R.run<OP_DOT>(p, q, S.pq);
            k_cols_alpha<<<cg, 256, 0, C.stream>>>(ld, S);
            k_axpy_xr<<<eg, 256, 0, C.stream>>>(total, ld, S.alpha, p, q, x, r);
            SSP_CHECK_LAUNCH();
            C.kernels_launched += 2;
            R.run<OP_SQ>(r, nullptr, S.rr);
            it++;
            SSP_CUDA(cudaMemsetAsync(nact, 0, sizeof(int64_t), C.stream));
            k_cols_check<<<cg, 256, 0, C.stream>>>(ld, it, S);
            SSP_CHECK_LAUNCH();
            C.kernels_launched++;
            active = read_i64(C, nact);
            if (opt.verbose && (it % 10 == 0 || active == 0))
                fprintf(stderr, "[ssp] pcg iter %d: %lld columns active\n", it, (long long)active);
            if (active == 0) break;
            ev_pc.begin(C.stream);
            SSP_CUDA(cudaGraphLaunch(P.exec, C.stream));
            ev_pc.end(C.stream);
            C.kernels_launched += pc_launches;
            R.run<OP_DOT>(r, z, S.rz_new);
            k_cols_beta<<<cg, 256, 0, C.stream>>>(ld, S);
            k_update_p<<<eg, 256, 0, C.stream>>>(total, ld, S.beta, z, p);
            SSP_CHECK_LAUNCH();
            C.kernels_launched += 2;
        }
    }
    // true relative residual ||b - A x|| / ||b||
    k_spmm<<<sgrid, 256, 0, C.stream>>>(n, lap_ptr, lap_idx, lap_val, x, q, ld);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    R.run<OP_SQDIFF>(b, q, relres);
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
    // x (ld) -> Zout (ldy)
    if (Zout != x) {
        SSP_CUDA(cudaMemcpy2DAsync(Zout, sizeof(double) * ldy, x, sizeof(double) * ld, sizeof(double) * k, n,
                                   cudaMemcpyDeviceToDevice, C.stream));
    }
}

}  // namespace ssp
