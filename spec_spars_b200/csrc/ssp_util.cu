// ssp_util.cu -- deterministic device-wide scans and segmented sorts used by the
// graph assembly and factorization stages.
#include <algorithm>
#include <cstring>
#include <thread>

#include "ssp_internal.cuh"
#include "ssp_sort.cuh"

namespace ssp {

// ---------------------------------------------------------------- scan
// Three-phase exclusive scan over int64 with 4096-element tiles.
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <class TIn>
__global__ void k_tile_sums(const TIn* in, int64_t n, int64_t* sums) {
    __shared__ int64_t warp_sums[32];
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    int64_t s = 0;
    for (int i = 0; i < SCAN_ITEMS; i++) {
        int64_t idx = base + (int64_t)i * SCAN_THREADS + threadIdx.x;
        if (idx < n) s += (int64_t)in[idx];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        int64_t t = warp_sums[threadIdx.x];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) sums[blockIdx.x] = t;
    }
}

// Scans one tile in shared memory; adds `offsets[blockIdx.x]` (if non-null).
template <class TIn>
__global__ void k_tile_scan(const TIn* in, int64_t* out, int64_t n, const int64_t* offsets, int64_t* total) {
    __shared__ int64_t warp_tot[32];
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    int64_t v[SCAN_ITEMS];
    int64_t run = 0;
    for (int i = 0; i < SCAN_ITEMS; i++) {
        int64_t idx = base + i;
        int64_t x = (idx < n) ? (int64_t)in[idx] : 0;
        v[i] = run;
        run += x;
    }
    // exclusive scan of `run` over the block
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int64_t incl = run;
    for (int o = 1; o < 32; o <<= 1) {
        int64_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int64_t t = warp_tot[lane];
        int64_t ti = t;
        for (int o = 1; o < 32; o <<= 1) {
            int64_t u = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o) ti += u;
        }
        warp_tot[lane] = ti - t;  // exclusive
        if (lane == 31 && total && offsets == nullptr && gridDim.x == 1) *total = ti;
    }
    __syncthreads();
    int64_t off = warp_tot[wid] + (incl - run) + (offsets ? offsets[blockIdx.x] : 0);
    for (int i = 0; i < SCAN_ITEMS; i++) {
        int64_t idx = base + i;
        if (idx < n) out[idx] = off + v[i];
    }
    if (total && offsets != nullptr && blockIdx.x == gridDim.x - 1 && threadIdx.x == SCAN_THREADS - 1) {
        *total = off + run;
    }
}

// nesting depth of the running scan on this thread, shared by every input type: an int32 scan recurses into
// the int64 one, and each level needs its own tile-sum buffer
static thread_local int g_scan_depth = 0;

template <class TIn>
static void scan_impl(Context& C, const TIn* in, int64_t* out, int64_t n, int64_t* d_total) {
    if (n <= 0) {
        if (d_total) SSP_CUDA(cudaMemsetAsync(d_total, 0, sizeof(int64_t), C.stream));
        return;
    }
    int64_t tiles = ceil_div<int64_t>(n, SCAN_TILE);
    if (tiles == 1) {
        k_tile_scan<TIn><<<1, SCAN_THREADS, 0, C.stream>>>(in, out, n, nullptr, d_total);
        SSP_CHECK_LAUNCH();
        C.kernels_launched++;
        return;
    }
    // tile sums are staged in a per-depth buffer: (in may alias out)
    int& depth = g_scan_depth;
    std::string tag = "scan_sums_" + std::to_string(depth);
    int64_t* sums = C.ws.get_t<int64_t>(tag, tiles + 1);
    k_tile_sums<TIn><<<(unsigned)tiles, SCAN_THREADS, 0, C.stream>>>(in, n, sums);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    depth++;
    try {
        scan_impl<int64_t>(C, sums, sums, tiles, nullptr);
    } catch (...) {
        depth--;
        throw;
    }
    depth--;
    k_tile_scan<TIn><<<(unsigned)tiles, SCAN_THREADS, 0, C.stream>>>(in, out, n, sums, d_total);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
}

void exclusive_scan_i64(Context& C, const int64_t* in, int64_t* out, int64_t n, int64_t* d_total) {
    scan_impl<int64_t>(C, in, out, n, d_total);
}
void exclusive_scan_i32_to_i64(Context& C, const int32_t* in, int64_t* out, int64_t n, int64_t* d_total) {
    scan_impl<int32_t>(C, in, out, n, d_total);
}

void make_chunks(const std::vector<int64_t>& ptr, int32_t r0, int32_t r1, std::vector<int32_t>& starts) {
    make_chunks(ptr.data(), r0, r1, starts);
}

void make_chunks(const int64_t* ptr, int32_t r0, int32_t r1, std::vector<int32_t>& starts) {
    int32_t r = r0;
    while (r < r1) {
        starts.push_back(r);
        int32_t e = r + 1;
        while (e < r1 && e - r < CHUNK_ROWS && ptr[e + 1] - ptr[r] <= CHUNK_CAP) e++;
        r = e;
    }
}

__global__ void k_max_offdiag_column(int64_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                     unsigned long long* mx) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long d = 0;
        for (int64_t p = ptr[c]; p < ptr[c + 1]; p++) d += idx[p] != c;
        atomicMax(mx, d);
    }
}

int64_t max_offdiag_column(Context& C, int64_t n, const int64_t* ptr, const int32_t* idx) {
    unsigned long long* d = C.ws.get_t<unsigned long long>("u_maxcol", 1);
    SSP_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), C.stream));
    if (n > 0) {
        k_max_offdiag_column<<<grid_for(n, 256), 256, 0, C.stream>>>(n, ptr, idx, d);
        SSP_CHECK_LAUNCH();
        C.kernels_launched++;
    }
    return read_i64(C, reinterpret_cast<const int64_t*>(d));
}

int64_t read_i64(Context& C, const int64_t* d_ptr) {
    SSP_CUDA(cudaMemcpyAsync(C.h_pinned, d_ptr, sizeof(int64_t), cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    return C.h_pinned[0];
}
void read_i64s(Context& C, const int64_t* d_ptr, int64_t* host, int cnt) {
    constexpr int PINNED = 64;  // entries of the context's pinned scratch
    for (int i0 = 0; i0 < cnt; i0 += PINNED) {
        const int c = std::min(PINNED, cnt - i0);
        SSP_CUDA(cudaMemcpyAsync(C.h_pinned, d_ptr + i0, sizeof(int64_t) * c, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
        for (int i = 0; i < c; i++) host[i0 + i] = C.h_pinned[i];
    }
}

// ---------------------------------------------------------------- segmented sort
struct KeyLessI32 {
    __device__ bool operator()(const int32_t& a, const int32_t& b) const { return a < b; }
};

// segments of length <= 32: one warp each, in registers
template <bool PAIRS>
__global__ void k_segsort_warp(int32_t* keys, double* vals, const int64_t* seg_start, const int32_t* seg_len,
                               int64_t nseg) {
    int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (w >= nseg) return;
    int32_t len = seg_len[w];
    if (len <= 1 || len > 32) return;
    int64_t s = seg_start[w];
    int32_t k = lane < len ? keys[s + lane] : INT32_MAX;
    double v = (PAIRS && lane < len) ? vals[s + lane] : 0.0;
    warp_bitonic_kv(k, v, lane, KeyLessI32());
    if (lane < len) {
        keys[s + lane] = k;
        if (PAIRS) vals[s + lane] = v;
    }
}

// segments longer than 32: one block each, bitonic over `cap` padded slots in shared memory
// (or in a global scratch slice when cap exceeds the shared budget).
template <bool PAIRS>
__global__ void k_segsort_block(int32_t* keys, double* vals, const int64_t* seg_start, const int32_t* seg_len,
                                const int32_t* list, int64_t nlist, int32_t cap, int32_t* gkeys, double* gvals) {
    extern __shared__ unsigned char smem[];
    for (int64_t li = blockIdx.x; li < nlist; li += gridDim.x) {
        int64_t sg = list[li];
        int32_t len = seg_len[sg];
        int64_t s = seg_start[sg];
        int P = 64;
        while (P < len) P <<= 1;
        int32_t* sk;
        double* sv;
        if (gkeys) {
            sk = gkeys + (int64_t)blockIdx.x * cap;
            sv = gvals + (int64_t)blockIdx.x * cap;
        } else {
            sv = (double*)smem;
            sk = (int32_t*)(smem + sizeof(double) * (size_t)(PAIRS ? cap : 0));
        }
        for (int i = threadIdx.x; i < P; i += blockDim.x) {
            sk[i] = i < len ? keys[s + i] : INT32_MAX;
            if (PAIRS) sv[i] = i < len ? vals[s + i] : 0.0;
        }
        __syncthreads();
        block_bitonic_kv<PAIRS>(sk, sv, P, KeyLessI32());
        for (int i = threadIdx.x; i < len; i += blockDim.x) {
            keys[s + i] = sk[i];
            if (PAIRS) vals[s + i] = sv[i];
        }
        __syncthreads();
    }
}

__global__ void k_seg_classify(const int32_t* seg_len, int64_t nseg, int32_t lim_smem, int32_t* list_mid,
                               int64_t* cnt_mid, int32_t* list_big, int64_t* cnt_big) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nseg; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t len = seg_len[i];
        if (len <= 32) continue;
        if (len <= lim_smem) list_mid[atomicAdd((unsigned long long*)cnt_mid, 1ull)] = (int32_t)i;
        else list_big[atomicAdd((unsigned long long*)cnt_big, 1ull)] = (int32_t)i;
    }
}

template <bool PAIRS>
static void segsort_impl(Context& C, int32_t* keys, double* vals, const int64_t* seg_start, const int32_t* seg_len,
                         int64_t nseg, int32_t max_len) {
    if (nseg <= 0 || max_len <= 1) return;
    {
        int threads = 256;
        int64_t blocks = ceil_div<int64_t>(nseg * 32, threads);
        k_segsort_warp<PAIRS><<<(unsigned)blocks, threads, 0, C.stream>>>(keys, vals, seg_start, seg_len, nseg);
        SSP_CHECK_LAUNCH();
        C.kernels_launched++;
    }
    if (max_len <= 32) return;
    const int32_t lim_smem = PAIRS ? 8192 : 16384;
    int32_t* list_mid = C.ws.get_t<int32_t>("segsort_mid", nseg);
    int32_t* list_big = C.ws.get_t<int32_t>("segsort_big", nseg);
    int64_t* cnts = C.ws.get_t<int64_t>("segsort_cnt", 2);
    SSP_CUDA(cudaMemsetAsync(cnts, 0, 2 * sizeof(int64_t), C.stream));
    k_seg_classify<<<grid_for(nseg, 256), 256, 0, C.stream>>>(seg_len, nseg, lim_smem, list_mid, cnts, list_big,
                                                               cnts + 1);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    int64_t hc[2];
    read_i64s(C, cnts, hc, 2);
    if (hc[0] > 0) {
        int32_t cap = 64;
        while (cap < std::min(max_len, lim_smem)) cap <<= 1;
        size_t smem = (size_t)cap * (sizeof(int32_t) + (PAIRS ? sizeof(double) : 0));
        SSP_CUDA(cudaFuncSetAttribute(k_segsort_block<PAIRS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        int blocks = (int)std::min<int64_t>(hc[0], 148 * 4);
        k_segsort_block<PAIRS><<<blocks, 512, smem, C.stream>>>(keys, vals, seg_start, seg_len, list_mid, hc[0],
                                                                cap, nullptr, nullptr);
        SSP_CHECK_LAUNCH();
        C.kernels_launched++;
    }
    if (hc[1] > 0) {
        int32_t cap = 64;
        while (cap < max_len) cap <<= 1;
        int blocks = (int)std::min<int64_t>(hc[1], 64);
        int32_t* gk = C.ws.get_t<int32_t>("segsort_gk", (size_t)cap * blocks);
        double* gv = PAIRS ? C.ws.get_t<double>("segsort_gv", (size_t)cap * blocks) : nullptr;
        k_segsort_block<PAIRS><<<blocks, 1024, 0, C.stream>>>(keys, vals, seg_start, seg_len, list_big, hc[1], cap,
                                                              gk, gv);
        SSP_CHECK_LAUNCH();
        C.kernels_launched++;
    }
}

void segsort_i32(Context& C, int32_t* keys, const int64_t* seg_start, const int32_t* seg_len, int64_t nseg,
                 int32_t max_len) {
    segsort_impl<false>(C, keys, nullptr, seg_start, seg_len, nseg, max_len);
}
void segsort_pairs_i32_f64(Context& C, int32_t* keys, double* vals, const int64_t* seg_start,
                           const int32_t* seg_len, int64_t nseg, int32_t max_len) {
    segsort_impl<true>(C, keys, vals, seg_start, seg_len, nseg, max_len);
}


// ---------------------------------------------------------------- stable LSD radix sort (64-bit keys)
// 8-bit digits.  Each block owns a tile of RS_TILE consecutive items: a histogram pass, a digit-major
// scan of the block histograms, and a scatter that ranks equal digits in item order (warp match masks,
// then a per-digit prefix over the block's warps), so items with equal keys keep their order.
namespace {
constexpr int RS_THREADS = 256;
constexpr int RS_ROUNDS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ROUNDS;
constexpr int RS_WARPS = RS_THREADS / 32;
}  // namespace

__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const uint64_t* __restrict__ keys, int64_t n, int shift,
                                                        int32_t* __restrict__ hist, int64_t nblocks) {
    __shared__ int32_t s_h[256];
    s_h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * RS_TILE;
    for (int r = 0; r < RS_ROUNDS; r++) {
        const int64_t i = base + r * RS_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&s_h[(keys[i] >> shift) & 255], 1);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = s_h[threadIdx.x];
}

__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const uint64_t* __restrict__ kin,
                                                           const int32_t* __restrict__ vin, uint64_t* __restrict__ kout,
                                                           int32_t* __restrict__ vout, int64_t n, int shift,
                                                           const int64_t* __restrict__ offs, int64_t nblocks,
                                                           unsigned long long* __restrict__ err) {
    __shared__ int64_t s_run[256];
    __shared__ int64_t s_wc[RS_WARPS][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    s_run[threadIdx.x] = offs[(int64_t)threadIdx.x * nblocks + blockIdx.x];
    for (int w = 0; w < RS_WARPS; w++) s_wc[w][threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * RS_TILE;
    const unsigned lt = (1u << lane) - 1u;
    for (int r = 0; r < RS_ROUNDS; r++) {
        const int64_t i = base + r * RS_THREADS + threadIdx.x;
        const bool valid = i < n;
        const uint64_t key = valid ? kin[i] : 0;
        const int d = valid ? (int)((key >> shift) & 255) : 256;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & lt);
        if (valid && rank == 0) s_wc[warp][d] = __popc(peers);
        __syncthreads();
        {
            const int t = threadIdx.x;
            int64_t run = s_run[t];
            for (int w = 0; w < RS_WARPS; w++) {
                const int64_t c = s_wc[w][t];
                s_wc[w][t] = run;
                run += c;
            }
            s_run[t] = run;
        }
        __syncthreads();
        if (valid) {
            const int64_t pos = s_wc[warp][d] + rank;
            if (pos >= 0 && pos < n) {
                kout[pos] = key;
                vout[pos] = vin[i];
            } else if (err) {
                atomicMin(err, (8ull << 48) | ((unsigned long long)i & ((1ull << 48) - 1)));
            }
        }
        __syncthreads();
        for (int w = 0; w < RS_WARPS; w++) s_wc[w][threadIdx.x] = 0;
        __syncthreads();
    }
}

void radix_sort_u64(Context& C, uint64_t* keys, int32_t* vals, int64_t n, int key_bits, uint64_t* tmp_keys,
                    int32_t* tmp_vals, unsigned long long* err) {
    if (n <= 1 || key_bits <= 0) return;
    const int64_t nblocks = ceil_div<int64_t>(n, RS_TILE);
    int32_t* hist = C.ws.get_t<int32_t>("rs_hist", (size_t)256 * nblocks);
    int64_t* offs = C.ws.get_t<int64_t>("rs_offs", (size_t)256 * nblocks);
    uint64_t *ka = keys, *kb = tmp_keys;
    int32_t *va = vals, *vb = tmp_vals;
    int passes = 0;
    for (int shift = 0; shift < key_bits; shift += 8, passes++) {
        k_rs_hist<<<(unsigned)nblocks, RS_THREADS, 0, C.stream>>>(ka, n, shift, hist, nblocks);
        SSP_CHECK_LAUNCH();
        exclusive_scan_i32_to_i64(C, hist, offs, 256 * nblocks, nullptr);
        k_rs_scatter<<<(unsigned)nblocks, RS_THREADS, 0, C.stream>>>(ka, va, kb, vb, n, shift, offs, nblocks, err);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += 2;
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    if (passes & 1) {
        SSP_CUDA(cudaMemcpyAsync(keys, ka, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, C.stream));
        SSP_CUDA(cudaMemcpyAsync(vals, va, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, C.stream));
    }
}

// ---------------------------------------------------------------- large host <-> device copies
// CUDA copies pageable memory through its own staging at one host memcpy's speed (11 GB/s measured on the
// B200 host, against 37-40 GB/s from pinned memory).  Here a 3 x 32 MB pinned ring takes the chunks: the
// host side of each chunk is copied by up to four threads while the previous chunk's DMA runs.
namespace {
constexpr size_t STAGE_CHUNK = 32u << 20;
constexpr int STAGE_SLOTS = 3;
constexpr size_t LARGE_COPY = 64u << 20;  // smaller copies stay plain cudaMemcpyAsync

void ensure_staging(Context& C) {
    if (C.h_stage) return;
    SSP_CUDA(cudaHostAlloc((void**)&C.h_stage, STAGE_CHUNK * STAGE_SLOTS, cudaHostAllocDefault));
    for (auto& e : C.stage_ev) SSP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}

void parallel_memcpy(char* dst, const char* src, size_t n) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int T = (int)std::min<unsigned>(4, hw);
    if (T <= 1 || n < (4u << 20)) {
        memcpy(dst, src, n);
        return;
    }
    const size_t part = (n / T + 4095) & ~(size_t)4095;
    std::thread th[4];
    for (int t = 1; t < T; t++) {
        const size_t a = std::min(n, part * t), b = std::min(n, part * (t + 1));
        if (a < b) th[t] = std::thread([=] { memcpy(dst + a, src + a, b - a); });
    }
    memcpy(dst, src, std::min(n, part));
    for (int t = 1; t < T; t++)
        if (th[t].joinable()) th[t].join();
}
}  // namespace

void copy_h2d(Context& C, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return;
    if (bytes < LARGE_COPY) {
        SSP_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, C.stream));
        return;
    }
    ensure_staging(C);
    size_t off = 0;
    for (int i = 0; off < bytes; i++) {
        const int slot = i % STAGE_SLOTS;
        const size_t n = std::min(STAGE_CHUNK, bytes - off);
        if (i >= STAGE_SLOTS) SSP_CUDA(cudaEventSynchronize(C.stage_ev[slot]));
        char* st = C.h_stage + (size_t)slot * STAGE_CHUNK;
        parallel_memcpy(st, (const char*)src + off, n);
        SSP_CUDA(cudaMemcpyAsync((char*)dst + off, st, n, cudaMemcpyHostToDevice, C.stream));
        SSP_CUDA(cudaEventRecord(C.stage_ev[slot], C.stream));
        off += n;
    }
    // the ring is reused by the next call; the caller's source is already free
    for (auto& e : C.stage_ev) SSP_CUDA(cudaEventSynchronize(e));
}

void copy_d2h(Context& C, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return;
    if (bytes < LARGE_COPY) {
        SSP_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
        return;
    }
    ensure_staging(C);
    const size_t nch = (bytes + STAGE_CHUNK - 1) / STAGE_CHUNK;
    auto issue = [&](size_t i) {
        const int slot = (int)(i % STAGE_SLOTS);
        const size_t off = i * STAGE_CHUNK, n = std::min(STAGE_CHUNK, bytes - off);
        SSP_CUDA(cudaMemcpyAsync(C.h_stage + (size_t)slot * STAGE_CHUNK, (const char*)src + off, n,
                                 cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaEventRecord(C.stage_ev[slot], C.stream));
    };
    for (size_t i = 0; i < nch && i < (size_t)STAGE_SLOTS; i++) issue(i);
    for (size_t i = 0; i < nch; i++) {
        const int slot = (int)(i % STAGE_SLOTS);
        const size_t off = i * STAGE_CHUNK, n = std::min(STAGE_CHUNK, bytes - off);
        SSP_CUDA(cudaEventSynchronize(C.stage_ev[slot]));
        parallel_memcpy((char*)dst + off, C.h_stage + (size_t)slot * STAGE_CHUNK, n);
        if (i + STAGE_SLOTS < nch) issue(i + STAGE_SLOTS);
    }
}

void release_staging(Context& C) {
    for (auto& e : C.stage_ev) {
        if (e) cudaEventDestroy(e);
        e = nullptr;
    }
    if (C.h_stage) cudaFreeHost(C.h_stage);
    C.h_stage = nullptr;
}

}  // namespace ssp
