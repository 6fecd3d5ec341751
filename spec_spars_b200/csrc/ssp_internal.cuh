// ssp_internal.cuh -- shared device/host helpers of the spec_spars B200 library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include <map>
#include <memory>
#include <stdexcept>
#include "../../include/specspars.h"

namespace ssp {

// ---------------------------------------------------------------- errors
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
void set_last_error(const std::string& msg);

#define SSP_CUDA(call)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            throw ::ssp::Error(SSP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
#define SSP_CHECK_LAUNCH() SSP_CUDA(cudaGetLastError())
#define SSP_REQUIRE(cond, code, msg)                       \
    do {                                                   \
        if (!(cond)) throw ::ssp::Error((code), (msg));    \
    } while (0)

// ---------------------------------------------------------------- RNG
// Philox4x64-10 (Salmon et al., SC'11).  Stream ids go into the second key word.
constexpr uint64_t STREAM_SIGN = 0x5349474eULL;
constexpr uint64_t STREAM_UNIF = 0x554e4946ULL;
constexpr uint64_t STREAM_FACTOR = 0x46414354ULL;
constexpr uint64_t STREAM_PRIO = 0x5052494fULL;
constexpr uint64_t STREAM_COIN = 0x434f494eULL;

struct u64x4 { uint64_t x, y, z, w; };

__host__ __device__ __forceinline__ uint64_t mulhi64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

__host__ __device__ __forceinline__ u64x4 philox(uint64_t c0, uint64_t c1, uint64_t c2, uint64_t c3,
                                                 uint64_t k0, uint64_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += 0x9E3779B97F4A7C15ULL;
            k1 += 0xBB67AE8584CAA73BULL;
        }
        const uint64_t M0 = 0xD2E7470EE14C6C93ULL, M1 = 0xCA5A826395121157ULL;
        uint64_t lo0 = M0 * c0, hi0 = mulhi64(M0, c0);
        uint64_t lo1 = M1 * c2, hi1 = mulhi64(M1, c2);
        uint64_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    return {c0, c1, c2, c3};
}
__host__ __device__ __forceinline__ uint64_t pick(const u64x4& r, int i) {
    return i == 0 ? r.x : i == 1 ? r.y : i == 2 ? r.z : r.w;
}
__host__ __device__ __forceinline__ double u53(uint64_t x) { return (double)(x >> 11) * 0x1.0p-53; }

__host__ __device__ __forceinline__ uint64_t vertex_priority(uint64_t seed, int64_t v) {
    return philox((uint64_t)v, 0, 0, 0, seed, STREAM_PRIO).x;
}
__host__ __device__ __forceinline__ double factor_uniform(uint64_t seed, int64_t v, int64_t slot) {
    u64x4 r = philox((uint64_t)v, (uint64_t)(slot >> 2), 0, 0, seed, STREAM_FACTOR);
    return u53(pick(r, (int)(slot & 3)));
}
__host__ __device__ __forceinline__ double edge_coin(uint64_t seed, int64_t e) {
    u64x4 r = philox((uint64_t)(e >> 2), 0, 0, 0, seed, STREAM_COIN);
    return u53(pick(r, (int)(e & 3)));
}

// ---------------------------------------------------------------- device memory
// Grow-only named buffers owned by a context, so repeated calls on one context do not allocate inside the hot
// loop.  Allocations and frees are stream-ordered (cudaMallocAsync / cudaFreeAsync on the context's stream,
// from the device's default memory pool): a buffer that grows, or a workspace that is released, never waits
// for the whole device the way cudaFree does, so contexts working side by side (the server's slots) do not
// stall each other.  The context's stream is the only stream that touches these buffers.
class Workspace {
public:
    ~Workspace() { release(); }
    // the stream allocations and frees are ordered on (the caller synchronizes the previous one first)
    void set_stream(cudaStream_t s) { stream_ = s; }
    void* get(const std::string& name, size_t bytes) {
        bytes = bytes ? bytes : 16;
        auto it = bufs_.find(name);
        if (it != bufs_.end() && it->second.bytes >= bytes) return it->second.ptr;
        if (it != bufs_.end()) {
            cudaFreeAsync(it->second.ptr, stream_);
            bufs_.erase(it);
        }
        void* p = nullptr;
        cudaError_t e = cudaMallocAsync(&p, bytes, stream_);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Error(SSP_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes for '" + name +
                                           "' failed: " + cudaGetErrorString(e));
        }
        bufs_[name] = {p, bytes};
        return p;
    }
    template <class T>
    T* get_t(const std::string& name, size_t count) { return (T*)get(name, count * sizeof(T)); }
    // enlarge `name` to `bytes`, preserving its first `keep` bytes
    void* grow(const std::string& name, size_t keep, size_t bytes, cudaStream_t stream) {
        auto it = bufs_.find(name);
        if (it != bufs_.end() && it->second.bytes >= bytes) return it->second.ptr;
        void* p = nullptr;
        cudaError_t e = cudaMallocAsync(&p, bytes, stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Error(SSP_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes for '" + name +
                                           "' failed: " + cudaGetErrorString(e));
        }
        if (it != bufs_.end()) {
            if (keep) {
                e = cudaMemcpyAsync(p, it->second.ptr, keep, cudaMemcpyDeviceToDevice, stream);
                if (e != cudaSuccess) {
                    cudaFreeAsync(p, stream);
                    throw Error(SSP_ERR_CUDA, std::string("workspace grow copy: ") + cudaGetErrorString(e));
                }
            }
            // ordered after the copy on the same stream
            cudaFreeAsync(it->second.ptr, stream);
            bufs_.erase(it);
        }
        bufs_[name] = {p, bytes};
        return p;
    }
    void release() {
        for (auto& kv : bufs_) cudaFreeAsync(kv.second.ptr, stream_);
        bufs_.clear();
    }
    size_t total_bytes() const {
        size_t s = 0;
        for (auto& kv : bufs_) s += kv.second.bytes;
        return s;
    }
    size_t bytes_with_prefix(const std::string& p) const {
        size_t s = 0;
        for (auto& kv : bufs_)
            if (kv.first.compare(0, p.size(), p) == 0) s += kv.second.bytes;
        return s;
    }
private:
    struct Buf { void* ptr; size_t bytes; };
    std::map<std::string, Buf> bufs_;
    cudaStream_t stream_ = nullptr;
};

// Launch shapes of the preconditioner's level launches (ssp_pcg.cu): per level and direction, the column width
// of a warp's row -- code 0, 1, 2 for 8, 16, 32 columns, TILE / width blocks per column tile.  Every width gives
// the same values bit for bit, so a shape changes only the time.  Chosen by measurement per factor and kept in
// the context under a signature of the factor's level structure and the solve's shape.
struct TrsvShapes {
    std::vector<uint8_t> fw, bw;  // per level
};
struct TrsvShapeCache {
    std::vector<std::pair<uint64_t, TrsvShapes>> entries;  // oldest first; a few graphs' worth
};

struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    Workspace ws;
    int64_t* h_pinned = nullptr;  // small pinned scratch for scalar readbacks
    // pinned staging ring for large copies between pageable host memory and the device (copy_*_large)
    char* h_stage = nullptr;
    cudaEvent_t stage_ev[3] = {nullptr, nullptr, nullptr};
    int verbose = 0;
    int64_t kernels_launched = 0;  // count of library kernel launches (for bench accounting)
    TrsvShapeCache trsv_cache;     // measured level-launch shapes of recently solved factors
};

// ---------------------------------------------------------------- n x k block layout
// Tile-major: k columns are split into tiles of SSP_TILE columns; each tile is a contiguous n x SSP_TILE
// slab, element (r, c) at ((c / SSP_TILE) * n + r) * SSP_TILE + c % SSP_TILE.  Kernels that gather rows
// work on one tile at a time.  32 columns make one gathered row 256 B in FP64 (128 B in FP32): a warp reads
// it whole and coalesced, and the sparse matrix is streamed once per 32 columns.  (Measured on B200 at
// ER n = 1M, k = 1327: 8-column tiles 69 ms per SpMM, 16 columns 62 ms, 32 columns 51 ms.)  Kernels assume
// SSP_TILE <= 32 (one warp lane per column).
#ifndef SSP_TILE_SHIFT
#define SSP_TILE_SHIFT 5
#endif
constexpr int SSP_TILE = 1 << SSP_TILE_SHIFT;
__host__ __device__ __forceinline__ int64_t tile_off(int64_t n, int64_t r, int64_t c) {
    return ((c >> SSP_TILE_SHIFT) * n + r) * SSP_TILE + (c & (SSP_TILE - 1));
}
__host__ __device__ __forceinline__ int64_t tile_ld(int64_t k) { return (k + SSP_TILE - 1) / SSP_TILE * SSP_TILE; }
// right-hand sides of the factor autotuner's probe solve: the first global columns of the sketch
constexpr int SSP_PROBE_COLS = 8;

// ---------------------------------------------------------------- small device helpers
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// One warp's sum over columns [0, k) of (Z[a, j] - Z[b, j])^2 (compute_diff_norms, sparsifier.rs:565-583),
// Z row-major with leading dimension ldz or (TM) tile-major with n rows.  Per 32-column group lane l squares
// the difference in column j0 + l (0 past k), a fixed xor butterfly sums the 32 squares and the groups are
// added in order; every lane returns the same value.  Every step is an explicit round-to-nearest operation,
// so the CPU oracle and every kernel that calls this form the same bits.
template <bool TM>
__device__ __forceinline__ double warp_edge_sq(int64_t a, int64_t b, const double* __restrict__ Z, int32_t k,
                                               int64_t ldz, int64_t n, int lane) {
    double acc = 0.0;
    for (int32_t j0 = 0; j0 < k; j0 += 32) {
        const int32_t j = j0 + lane;
        double x = 0.0;
        if (j < k) {
            const int64_t oa = TM ? tile_off(n, a, j) : a * ldz + j;
            const int64_t ob = TM ? tile_off(n, b, j) : b * ldz + j;
            x = __dsub_rn(Z[oa], Z[ob]);
        }
        double s = __dmul_rn(x, x);
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) s = __dadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
        acc = __dadd_rn(acc, s);
    }
    return acc;
}

// p_e = min(((beta * w_e) * d_e^2) / denom, 1) (compute_probs, sparsifier.rs:542-562); a NaN ratio (an edge
// whose norm could not be formed) maps to 1, so such an edge is always kept.
__device__ __forceinline__ double leverage_prob(double w, double d, double beta, double denom) {
    const double d2 = __dmul_rn(d, d);
    const double x = __ddiv_rn(__dmul_rn(__dmul_rn(beta, w), d2), denom);
    if (x != x) return 1.0;
    return (x < 1.0) ? x : 1.0;
}

template <class T>
inline T ceil_div(T a, T b) { return (a + b - 1) / b; }

inline int grid_for(int64_t items, int per_block, int max_blocks = 148 * 32) {
    int64_t g = (items + per_block - 1) / per_block;
    if (g < 1) g = 1;
    if (g > max_blocks) g = max_blocks;
    return (int)g;
}

// Device-wide exclusive scan of int64 counts (three-phase, deterministic).
// out may alias in.  Returns total via *d_total (device) if non-null.
void exclusive_scan_i64(Context& C, const int64_t* in, int64_t* out, int64_t n, int64_t* d_total);
void exclusive_scan_i32_to_i64(Context& C, const int32_t* in, int64_t* out, int64_t n, int64_t* d_total);

// read a device scalar synchronously (on the context stream)
int64_t read_i64(Context& C, const int64_t* d_ptr);
void read_i64s(Context& C, const int64_t* d_ptr, int64_t* host, int cnt);

// Row-aligned chunks of a CSR row range: each holds at most CHUNK_CAP entries and CHUNK_ROWS rows
// (a longer row is a chunk of its own).  Appends chunk starts for rows [r0, r1).
#ifndef SSP_CHUNK_CAP
#define SSP_CHUNK_CAP 256
#endif
constexpr int CHUNK_CAP = SSP_CHUNK_CAP;
constexpr int CHUNK_ROWS = 32;
void make_chunks(const std::vector<int64_t>& ptr, int32_t r0, int32_t r1, std::vector<int32_t>& starts);
void make_chunks(const int64_t* ptr, int32_t r0, int32_t r1, std::vector<int32_t>& starts);
// Copies between pageable host memory and the device on C.stream, returning once the host side is done
// (host to device: the source may be reused; device to host: the data is in dst).  Large copies go through
// a pinned staging ring with the host-side memcpy split over a few threads and overlapped with the DMA;
// small ones are plain cudaMemcpyAsync.
void copy_h2d(Context& C, void* dst, const void* src, size_t bytes);
void copy_d2h(Context& C, void* dst, const void* src, size_t bytes);
void release_staging(Context& C);
// Matrix Market on the device (ssp_mtxio.cu).  read_mtx_device leaves the CSC in workspace buffers named
// after tag and returns false when the file needs the host reader; write_mtx_device takes device arrays.
bool read_mtx_device(Context& C, const char* path, int64_t* n, int64_t* nnz, int64_t** colptr, int32_t** rowidx,
                     double** val, const std::string& tag);
void write_mtx_device(Context& C, const char* path, int64_t n, const int64_t* colptr, const int32_t* rowidx,
                      const double* val, const std::string& tag);
// edge list -> .mtx on the device; false when the host converter must run (it then gives the same result)
bool edgelist_to_mtx_device(Context& C, const char* in_path, const char* out_path, double default_weight);
// stable ascending sort of (key, value) pairs by the low key_bits bits of the keys (LSD radix, 8-bit digits);
// tmp_* are scratch arrays of n items; a scatter outside [0, n) is skipped and recorded in *err (if given)
void radix_sort_u64(Context& C, uint64_t* keys, int32_t* vals, int64_t n, int key_bits, uint64_t* tmp_keys,
                    int32_t* tmp_vals, unsigned long long* err = nullptr);
// L2 share (MB) of one column slab of the PCG's Laplacian product (SSP_SPMM_SLAB_MB; 0 = one pass)
double spmm_slab_mb();

// Segmented sort of int32 keys in place (ascending).  Segments [start[i], start[i]+len[i]).
void segsort_i32(Context& C, int32_t* keys, const int64_t* seg_start, const int32_t* seg_len, int64_t nseg,
                 int32_t max_len);
// Segmented sort of (int32 key, double payload) pairs by key (keys unique within a segment).
void segsort_pairs_i32_f64(Context& C, int32_t* keys, double* vals, const int64_t* seg_start,
                           const int32_t* seg_len, int64_t nseg, int32_t max_len);

// ---------------------------------------------------------------- stage entry points (internal C++)
struct DevGraph {
    int64_t n = 0, m = 0;
    int32_t *v1 = nullptr, *v2 = nullptr;  // edges in reference order
    double* w = nullptr;
    int64_t* adj_ptr = nullptr;            // [n+1] symmetric adjacency, neighbour-sorted
    int32_t* adj_nbr = nullptr;            // [2m]
    int32_t* adj_eid = nullptr;            // [2m]
    int32_t max_deg = 0;
    // Laplacian L_G (CSC == CSR)
    int64_t lap_nnz = 0;
    int64_t* lap_ptr = nullptr;
    int32_t* lap_idx = nullptr;
    double* lap_val = nullptr;
    int32_t* lap_eid = nullptr;  // [lap_nnz] edge of an entry with row < column, else -1
};

// a2+a5: build edges, adjacency and L_G from an input CSC already on the device.
// tag prefixes the workspace buffers, so that two graphs can be held at once
void build_graph_from_csc(Context& C, int64_t n, const int64_t* colptr, const int32_t* rowidx,
                          const double* val, int64_t nnz, DevGraph& G, const std::string& tag = "g");
// the graph of a device Laplacian: its off-diagonal entries negated, in stored order (workspace buffers
// tag_ptr/_idx/_val); returns the graph's nnz
int64_t laplacian_to_graph_device(Context& C, int64_t n, int64_t nnz, const int64_t* ptr, const int32_t* idx,
                                  const double* val, int64_t** gptr, int32_t** gidx, double** gval,
                                  const std::string& tag = "lapg");
// adjacency + Laplacian for a given device edge list (v1<v2, CSC order)
void build_graph_from_edges(Context& C, DevGraph& G, const std::string& tag = "g");

// the current Laplacian's off-diagonals as a graph plus a batch of new edges (a symmetric CSC), duplicates
// summed; returns nnz of the merged graph CSC, left in workspace buffers
int64_t laplacian_plus_graph_device(Context& C, int64_t n, const int64_t* lptr, const int32_t* lidx,
                                    const double* lval, const int64_t* bptr, const int32_t* bidx, const double* bval,
                                    int64_t** mptr, int32_t** midx, double** mval);

// a4: Y = B^T Q, columns [0,k): row-major with leading dimension ldy, or tile-major (SSP_TILE-column slabs)
void sketch_device(Context& C, const DevGraph& G, int32_t k, double scale, uint64_t seed, int uniform,
                   double* Y, int64_t ldy, int tile_major, int32_t col_lo = 0);
// the same for vertices [v0, v0 + nv) only, edge ids counted from e0 (one graph of a union of graphs)
void sketch_device_part(Context& C, const DevGraph& G, int64_t v0, int64_t nv, int64_t e0, int32_t k, double scale,
                        uint64_t seed, int uniform, double* Y, int64_t ldy, int tile_major, int32_t col_lo = 0);

// a7: factor
struct DevFactor {
    int64_t n = 0;
    int64_t nnz = 0;
    // column form (backward solve): vertex-indexed CSC
    int64_t* col_ptr = nullptr;
    int32_t* col_idx = nullptr;
    double* col_val = nullptr;
    // row form (forward solve): vertex-indexed CSR, columns sorted
    int64_t* row_ptr = nullptr;
    int32_t* row_idx = nullptr;
    double* row_val = nullptr;
    double* D = nullptr;
    int32_t* level = nullptr;       // [n]
    int32_t* level_ptr_d = nullptr; // [num_levels+1] (device)
    int32_t* level_rows = nullptr;  // [n] vertices grouped by level ("storage order")
    std::vector<int32_t> level_ptr; // host copy
    // L rows (forward solve) and columns (backward solve) re-laid in storage order, so that the rows of
    // a level are contiguous; chunk lists split each level into row-aligned pieces of bounded size
    int64_t* prow_ptr = nullptr;
    int32_t* prow_idx = nullptr;
    double* prow_val = nullptr;
    int64_t* pcol_ptr = nullptr;
    int32_t* pcol_idx = nullptr;
    double* pcol_val = nullptr;
    int32_t* fchunk = nullptr;           // device chunk starts (storage rows) for the forward solve
    int32_t* bchunk = nullptr;           // ... for the backward solve
    std::vector<int32_t> fchunk_lvl;     // [num_levels+1] chunk index range per level
    std::vector<int32_t> bchunk_lvl;
    int32_t num_levels = 0;
    int32_t dense_levels = 0;       // trailing single-vertex levels from the dense phase
    int32_t max_level_rows = 0;
    std::vector<int64_t> frontier_sizes;  // rows of each sparse level
    int32_t compactions = 0;
    int64_t truncated_rows = 0;           // vertices left to the diagonal final level
    // entries of the last level's rows in the row form (forward solve) and the column form (backward
    // solve); -1 until the storage-order forms are built.  The column count is 0 for every factor (nothing is
    // eliminated after the last level, and a level's rows never reference each other), which lets the
    // forward solve of that level finish its rows (z = y / D) and the backward solve skip it.
    int64_t last_fwd_nnz = -1;
    int64_t last_bwd_nnz = -1;
    // Solve schedule.  Maximal runs of consecutive thin levels (at most THIN_ROWS rows each, two or more
    // levels) are solved by one launch that walks "steps": the run's rows grouped by their dependency depth
    // inside the run (a row's depth is one more than the deepest row of the same run it reads), which is
    // often far smaller than the run's level count (the dense tail eliminates one vertex per level).  The
    // factor and its levels are unchanged; only the order rows are solved in differs, and each row's own
    // sum is formed the same way whatever step it lands in.
    struct SolveRun {
        int32_t l0, l1;  // levels [l0, l1)
        int32_t fs0, fs1, bs0, bs1;  // step ranges of the forward and backward schedules
    };
    std::vector<SolveRun> runs;
    int32_t* fsched = nullptr;  // storage rows of all runs, forward step order
    int32_t* fstep = nullptr;   // step pointers into fsched
    int32_t* bsched = nullptr;
    int32_t* bstep = nullptr;
};
constexpr int THIN_ROWS = 64;  // a level with at most this many rows is "thin"
struct FactorOptions {
    uint64_t seed = 0;
    int64_t dense_threshold = 4096;
    int64_t max_degree = 0;  // stop once the live Schur complement's average degree exceeds this (0: never)
    const int32_t* vbase = nullptr;  // device [n]: first vertex of each vertex's graph (several graphs at once)
    const int32_t* vseg = nullptr;   // device [n]: graph of each vertex; with max_degree > 0 each graph is
                                     // truncated by its own test, at the level where it would stop alone
    std::vector<int64_t> seg_row0;   // host: nseg + 1 first vertices of the graphs (with vseg)
    std::vector<int64_t> seg_max_degree;  // host: each graph's own truncation (with vseg; empty: max_degree)
};
// Input: Laplacian CSC on device (rows > col used, |value| as weight).
void factor_device(Context& C, int64_t n, const int64_t* colptr, const int32_t* rowidx, const double* val,
                   const FactorOptions& opt, DevFactor& F, const std::string& tag = "f");

// a8: PCG on all k columns.  Y: tile-major n x round8(k) device block; the solution is left in the
// workspace (tile-major) and returned through *x_out.
// Several graphs solved at once as the disjoint union of their Laplacians (rows [row0[s], row0[s + 1]) are
// graph s, which uses the first k[s] columns).  Every per-column scalar of the PCG is then per (graph,
// column), so each graph's iterates are its own.  iters / relres come back per (graph, column), at s * ld + c.
struct PcgSegments {
    std::vector<int64_t> row0;        // nseg + 1 row starts
    std::vector<int32_t> k;           // columns of each graph
    const int32_t* rowseg = nullptr;  // device [n]: graph of each row
    std::vector<int32_t> iters;       // out
    std::vector<double> relres;       // out
    // with record_history: per graph, per iteration, the largest ||r|| / ||b|| over its columns (the autotuner's
    // probe, graph by graph)
    bool record_history = false;
    std::vector<std::vector<double>> history;
};
struct PcgOptions {
    double tol = 1e-8;
    double abs_tol = 0.0;
    int32_t max_iters = 400;
    int verbose = 0;
    std::vector<double>* history = nullptr;  // per iteration: max over columns of ||r|| / ||b||
    int precision = SSP_PRECISION_FP64;      // SSP_PRECISION_MIXED: FP32 inner solves, FP64 refinement
    PcgSegments* segs = nullptr;             // several graphs at once (see PcgSegments)
};
struct PcgReport {
    int32_t max_iters_used = 0;
    double mean_iters = 0;
    double max_relres = 0;
    int32_t not_converged = 0;
    double ms_spmm = 0;
    int64_t n_spmm = 0;
    double ms_precond = 0;
    int64_t n_precond = 0;
    double ms_loop = 0;      // device time of the iteration loop
    int32_t iters_run = 0;   // iterations of the loop (all columns)
    int32_t refinements = 0; // mixed precision: outer rounds (true FP64 residual recomputations)
    int32_t fp64_rounds = 0; // mixed precision: rounds that fell back to an FP64 inner solve
    int32_t spmm_slabs = 1;  // column slabs of the Laplacian product
    double ms_resid = 0;     // mixed precision: device time of the FP64 residual products
    int64_t n_resid = 0;
    bool diff_fused = false; // the squared diff norms were formed by the final product (d2 filled)
    // level-launch shapes of the preconditioner (the last one built): SSP_TRSV_* source, level launches
    // (forward + backward) at 8, 16 and 32 columns per warp row, device time spent measuring them
    int32_t trsv_shapes = 0;
    int32_t trsv_levels[3] = {0, 0, 0};
    double ms_trsv_tune = 0;
};
// Picks the elimination truncation (FactorOptions::max_degree) for this Laplacian and right-hand sides
// by factoring a few candidates and timing a short PCG probe on the first column tile of Y.  Leaves
// the chosen factor in F and returns the chosen max_degree.
int64_t autotune_factor(Context& C, int64_t n, const int64_t* lap_ptr, const int32_t* lap_idx,
                        const double* lap_val, int64_t lap_offdiag_nnz, int64_t max_vertex_degree,
                        const double* Ytiles, int32_t k, const FactorOptions& base, const PcgOptions& popt,
                        DevFactor& F, double* ms_tuning);
// The autotuner's rule, its pieces shared by the single-graph and the batched autotuning: the lightest
// truncation for a graph of n vertices and lap_offdiag_nnz off-diagonal Laplacian entries, and the
// iterations to the tolerance predicted from a probe's residual history (1e9: no prediction).
int64_t autotune_light_degree(int64_t n, int64_t lap_offdiag_nnz);
double autotune_predicted_iters(const std::vector<double>& hist, double tol);
// whether the light factor is kept, given its predicted iterations and the graph's degrees
bool autotune_keep_light(double predicted_iters, int64_t n, int64_t lap_offdiag_nnz, int64_t max_vertex_degree);
// largest off-diagonal entry count of a column of a Laplacian (its largest vertex degree)
int64_t max_offdiag_column(Context& C, int64_t n, const int64_t* ptr, const int32_t* idx);
constexpr int32_t SSP_TUNE_PROBE_ITERS = 20;
constexpr double SSP_TUNE_MAX_ITERS = 30.0;
// With lap_eid (the graph's per-entry edge map) and d2 (m doubles), the final product A x also forms
// d2[e] = sum over columns of (x[v1_e] - x[v2_e])^2 in the order of diff_norms_device (per 32-column tile a
// butterfly over the tile's columns, tiles added in order) from the rows it gathers anyway, and sets
// rep.diff_fused; without them, or with a slab plan, d2 is left alone.
void pcg_device(Context& C, int64_t n, const int64_t* lap_ptr, const int32_t* lap_idx, const double* lap_val,
                const DevFactor& F, const double* Y, int32_t k, const double** x_out, const PcgOptions& opt,
                PcgReport& rep, int32_t* h_iters = nullptr, double* h_relres = nullptr,
                const int32_t* lap_eid = nullptr, double* d2 = nullptr, bool d2_accumulate = false);
void rowmajor_to_tiles(Context& C, int64_t n, int32_t k, int64_t ldr, const double* src, double* dst);
void tiles_to_rowmajor(Context& C, int64_t n, int32_t k, const double* src, double* dst, int64_t ldr);
void precond_apply_device(Context& C, const DevFactor& F, const double* R, double* Z, int64_t ld);

// a9-a12
// Z has n rows, row-major (leading dimension ldz) or tile-major; an edge with an endpoint outside [0, n) is
// not read and gets d = NaN
void diff_norms_device(Context& C, int64_t m, const int32_t* v1, const int32_t* v2, const double* Z, int32_t k,
                       int64_t ldz, double* d, int64_t n, bool tile_major);
// per-edge sum over the k columns of (Z[v1,j] - Z[v2,j])^2, Z tile-major with n_tile_major rows
void diff_sq_device(Context& C, int64_t m, const int32_t* v1, const int32_t* v2, const double* Z, int32_t k,
                    int64_t n_tile_major, double* sq);
void sqrt_device(Context& C, int64_t m, const double* sq, double* d);
// dst[i] += src[i]
void add_device(Context& C, int64_t m, const double* src, double* dst);
void probs_device(Context& C, int64_t m, const double* w, const double* d, double beta, double denom, double* p);
void coins_device(Context& C, int64_t m, uint64_t seed, double* coins);

// a15: checks (ssp_quality.cu)
void laplacian_check_device(Context& C, int64_t n, const int64_t* ptr, const int32_t* idx, const double* val,
                            double tol, int64_t* bad_cols, double* max_abs_colsum, int64_t* asym_entries);
void probe_vectors_device(Context& C, int64_t n, int32_t p, uint64_t seed, double* X);
void quadratic_forms_device(Context& C, int64_t n, const int64_t* ptr, const int32_t* idx, const double* val,
                            const double* X, int32_t p, double* out);
int64_t components_device(Context& C, int64_t n, const int64_t* ptr, const int32_t* idx, const double* val,
                          int32_t* labels);
// returns nnz(L_H); writes L_H CSC into workspace buffers returned through pointers
int64_t sample_apply_device(Context& C, const DevGraph& G, const double* p, const double* coins, int reweight,
                            int64_t** lh_ptr, int32_t** lh_idx, double** lh_val, uint8_t* keep_out);

}  // namespace ssp
