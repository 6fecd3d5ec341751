// ssp_factor.cu -- a7: randomized approximate Cholesky of a graph Laplacian on the device.
//
// Per-column arithmetic restates perform_factorization_device (example.cc:188-300): the entries
// of the column (original lower entries plus fill) are merged by row (:209-235), sorted by value
// (:243) and prefix-summed (:248-258); every entry but the last picks a partner j > i with
// probability proportional to weight (:264-268) and emits fill (max(r_i,r_j), min(r_i,r_j)) of
// weight v_i (S - c_i) / S (:269-271); L entries are -v_i / S (:293, :437-446), D = S (:441).
//
// Schedule (this build): vertices are eliminated in increasing (Philox priority, id) order.  A
// vertex is ready once every neighbour with a smaller key has been eliminated, which is the
// reference's dependency-count scheme (example.cc:163-168,302-315) with a random instead of the
// natural order.  Every ready vertex of a level is eliminated in parallel; they are pairwise
// non-adjacent, so the factor equals sequential elimination in key order.  Once at most
// `dense_threshold` vertices are live at a level boundary, the live Schur complement is merged into
// a dense matrix and eliminated one vertex per level by a single block.  (The switch also waits for the
// frontier to collapse to at most 8 vertices, so sparse Schur complements stay in the sparse phase.)
//
// Every random draw is Philox(seed, column, slot); merges sort by (row, weight) and sum runs
// left to right; prefix sums are 32-wide Kogge-Stone chunks with a sequential carry.  Compiled
// with -fmad=false, so results are bit-identical to the CPU oracle.
#include "ssp_internal.cuh"
#include "ssp_sort.cuh"

namespace ssp {

enum { C_NEXT = 0, C_LCUR, C_FCUR, C_ERR, C_NB, C_NG, C_MAXLIVE, C_POOL, C_OWNERS, C_REM, C_NFILL, C_NCTR };
enum { FERR_POOL = 1, FERR_OVERFLOW = 2 };
enum { GC_FCUR = 0, GC_NFRONT = 1, GC_NFILL = 2 };

constexpr int BLOCK_TIER_MAX = 4096;    // live entries handled in shared memory
constexpr int DENSE_FRONTIER_MAX = 8;   // dense tail once the frontier has collapsed to this size

struct FDev {
    int64_t n;
    uint64_t seed;
    // several graphs factored at once: vbase[v] is the first vertex of v's graph, and every random draw is keyed
    // by the vertex's id inside its graph, so each graph's factor is the one it gets alone (null: one graph)
    const int32_t* vbase;
    // ... and vseg[v] its graph: per graph, gctr[3 g + GC_*] count the upcoming frontier's live entries and
    // vertices and the fill of the level just eliminated, for the truncation test of each graph
    const int32_t* vseg;
    int64_t* gctr;
    int32_t nseg;
    const uint64_t* prio;
    int32_t* count;
    int32_t* level;
    int64_t* bag_start;
    int32_t* bag_len;
    int32_t* bag_cap;
    int32_t* pool_u;
    double* pool_w;
    int64_t pool_cap;
    int64_t* ctr;
    int64_t* Lstart;
    int32_t* Lcnt;
    int32_t* Lrow;
    double* Lval;
    double* D;
    // per-level frontier data
    int64_t* fstart;  // [frontier idx] fill region start
    int32_t* fcnt;    // [frontier idx] fills emitted
    int32_t* fill_a;
    int32_t* fill_b;
    double* fill_w;
};

__device__ __forceinline__ bool key_less(const uint64_t* prio, int32_t a, int32_t b) {
    uint64_t pa = prio[a], pb = prio[b];
    return pa != pb ? pa < pb : a < b;
}

// ---------------------------------------------------------------- init
__device__ __forceinline__ int64_t local_vertex(const int32_t* vbase, int64_t v) { return vbase ? v - vbase[v] : v; }

__global__ void k_prio(int64_t n, uint64_t seed, uint64_t* prio, const int32_t* vbase) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        prio[v] = vertex_priority(seed, local_vertex(vbase, v));
}

// lower entries (r > c, |val| != 0) counted for both endpoints
__global__ void k_lower_deg(int64_t n, const int64_t* colptr, const int32_t* rowidx, const double* val, int32_t* deg) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        int32_t cnt = 0;
        for (int64_t p = colptr[c]; p < colptr[c + 1]; p++) {
            int32_t r = rowidx[p];
            if (r > c && fabs(val[p]) != 0.0) {
                cnt++;
                atomicAdd(&deg[r], 1);
            }
        }
        atomicAdd(&deg[c], cnt);
    }
}

__global__ void k_bag_caps(int64_t n, const int32_t* deg, int32_t* cap) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        cap[v] = 2 * deg[v] + 4;
}

__global__ void k_bag_fill(int64_t n, const int64_t* colptr, const int32_t* rowidx, const double* val, FDev F) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        for (int64_t p = colptr[c]; p < colptr[c + 1]; p++) {
            int32_t r = rowidx[p];
            double w = fabs(val[p]);
            if (r > c && w != 0.0) {
                int32_t s1 = atomicAdd(&F.bag_len[c], 1);
                F.pool_u[F.bag_start[c] + s1] = r;
                F.pool_w[F.bag_start[c] + s1] = w;
                int32_t s2 = atomicAdd(&F.bag_len[r], 1);
                F.pool_u[F.bag_start[r] + s2] = (int32_t)c;
                F.pool_w[F.bag_start[r] + s2] = w;
            }
        }
    }
}

// warp per vertex: count entries pointing to smaller keys; ready vertices form the first frontier
__global__ void k_init_count(FDev F, int32_t* frontier) {
    int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = warp; v < F.n; v += nw) {
        int32_t cnt = 0;
        int64_t s = F.bag_start[v];
        int32_t len = F.bag_len[v];
        for (int32_t i = lane; i < len; i += 32) cnt += key_less(F.prio, F.pool_u[s + i], (int32_t)v) ? 1 : 0;
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == 0) {
            F.count[v] = cnt;
            F.level[v] = -1;
            if (cnt == 0) frontier[atomicAdd((unsigned long long*)&F.ctr[C_NEXT], 1ull)] = (int32_t)v;
        }
    }
}

// warp per frontier vertex: live entries, L and fill reservations, tier lists
__global__ void k_live_count(FDev F, const int32_t* frontier, int32_t* live_cnt, int32_t* list_b, int32_t* list_g) {
    int64_t nf = F.ctr[C_NEXT];
    int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < nf; i += nw) {
        int32_t v = frontier[i];
        int64_t s = F.bag_start[v];
        int32_t len = F.bag_len[v];
        int32_t cnt = 0;
        for (int32_t q = lane; q < len; q += 32) cnt += (F.level[F.pool_u[s + q]] < 0) ? 1 : 0;
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == 0) {
            live_cnt[i] = cnt;
            if (F.vseg) {
                atomicAdd((unsigned long long*)&F.gctr[3 * F.vseg[v] + GC_FCUR], (unsigned long long)cnt);
                atomicAdd((unsigned long long*)&F.gctr[3 * F.vseg[v] + GC_NFRONT], 1ull);
            }
            F.Lstart[v] = (int64_t)atomicAdd((unsigned long long*)&F.ctr[C_LCUR], (unsigned long long)cnt);
            F.fstart[i] = (int64_t)atomicAdd((unsigned long long*)&F.ctr[C_FCUR], (unsigned long long)cnt);
            atomicMax((unsigned long long*)&F.ctr[C_MAXLIVE], (unsigned long long)cnt);
            if (cnt > 32 && cnt <= BLOCK_TIER_MAX)
                list_b[atomicAdd((unsigned long long*)&F.ctr[C_NB], 1ull)] = (int32_t)i;
            else if (cnt > BLOCK_TIER_MAX)
                list_g[atomicAdd((unsigned long long*)&F.ctr[C_NG], 1ull)] = (int32_t)i;
        }
    }
}

// ---------------------------------------------------------------- elimination (shared tail)
// Given merged entries (mu, mw)[0..cnt) sorted by (w, u) and inclusive prefix sums sc, emit one slot.
__device__ __forceinline__ void emit_slot(const FDev& F, int32_t v, int64_t fidx, int32_t i, int32_t cnt,
                                          const int32_t* mu, const double* mw, const double* sc, double S) {
    const int64_t Ls = F.Lstart[v];
    F.Lrow[Ls + i] = mu[i];
    F.Lval[Ls + i] = -(mw[i] / S);
    if (i + 1 < cnt) {
        const double ci = sc[i];
        const double rem = S - ci;
        const double tgt = factor_uniform(F.seed, local_vertex(F.vbase, v), i) * rem;
        int32_t lo = i + 1, hi = cnt;
        while (lo < hi) {
            int32_t mid = lo + ((hi - lo) >> 1);
            if ((sc[mid] - ci) < tgt) lo = mid + 1;
            else hi = mid;
        }
        const int32_t j = lo < cnt ? lo : cnt - 1;
        const int32_t r0 = mu[i], r1 = mu[j];
        const int32_t a = r0 > r1 ? r0 : r1, b = r0 > r1 ? r1 : r0;
        const double wf = (mw[i] * rem) / S;
        if (fidx >= 0) {
            const int64_t fp = F.fstart[fidx] + i;
            F.fill_a[fp] = a;
            F.fill_b[fp] = b;
            F.fill_w[fp] = wf;
            atomicAdd(&F.count[key_less(F.prio, b, a) ? a : b], 1);
        }
    }
}

// Warp tier: <= 32 live entries, all in registers.
__global__ void __launch_bounds__(128) k_elim_warp(FDev F, const int32_t* frontier, const int32_t* live_cnt) {
    const int64_t nf = F.ctr[C_REM];  // frontier size of this level
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t fi = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; fi < nf; fi += nw) {
        const int32_t L = live_cnt[fi];
        if (L > 32) continue;
        const int32_t v = frontier[fi];
        const int64_t s = F.bag_start[v];
        const int32_t len = F.bag_len[v];
        // gather live entries (order irrelevant: sorted next) through a per-warp staging area
        __shared__ int32_t s_mu[4][32];
        __shared__ double s_mw[4][32];
        __shared__ double s_c[4][32];
        const int wib = threadIdx.x >> 5;
        int32_t got = 0;
        for (int32_t q0 = 0; q0 < len; q0 += 32) {
            int32_t q = q0 + lane;
            int32_t uu = 0;
            double ww = 0;
            bool live = false;
            if (q < len) {
                uu = F.pool_u[s + q];
                ww = F.pool_w[s + q];
                live = F.level[uu] < 0;
            }
            unsigned mask = __ballot_sync(0xffffffffu, live);
            if (live) {
                int32_t pos = got + __popc(mask & ((1u << lane) - 1u));
                if (pos < 32) {
                    s_mu[wib][pos] = uu;
                    s_mw[wib][pos] = ww;
                } else {
                    atomicOr((unsigned long long*)&F.ctr[C_ERR], (unsigned long long)FERR_OVERFLOW);
                }
            }
            got += __popc(mask);
        }
        got = got < 32 ? got : 32;
        __syncwarp();
        int32_t u = lane < got ? s_mu[wib][lane] : INT32_MAX;
        double w = lane < got ? s_mw[wib][lane] : __longlong_as_double(0x7ff0000000000000ll);
        __syncwarp();
        if (got == 0) {
            if (lane == 0) {
                F.D[v] = 0.0;
                F.Lcnt[v] = 0;
                F.fcnt[fi] = 0;
            }
            continue;
        }
        warp_bitonic_ent(u, w, lane, EntUW());
        // merge runs of equal u: the head lane sums its run left to right
        const int32_t prev_u = __shfl_up_sync(0xffffffffu, u, 1);
        const bool head = (lane < got) && (lane == 0 || prev_u != u);
        double sum = w;
        bool cont = true;
        for (int t = 1; t < 32; t++) {
            double ow = __shfl_down_sync(0xffffffffu, w, t);
            int32_t ou = __shfl_down_sync(0xffffffffu, u, t);
            if (cont && lane + t < got && ou == u) sum = sum + ow;
            else cont = false;
        }
        const unsigned hmask = __ballot_sync(0xffffffffu, head);
        const int32_t cnt = __popc(hmask);
        if (head) {
            int32_t pos = __popc(hmask & ((1u << lane) - 1u));
            s_mu[wib][pos] = u;
            s_mw[wib][pos] = sum;
        }
        __syncwarp();
        int32_t mu = lane < cnt ? s_mu[wib][lane] : INT32_MAX;
        double mw = lane < cnt ? s_mw[wib][lane] : __longlong_as_double(0x7ff0000000000000ll);
        __syncwarp();
        warp_bitonic_ent(mu, mw, lane, EntWU());
        // 32-wide Kogge-Stone inclusive scan (lanes >= cnt hold 0)
        double c = lane < cnt ? mw : 0.0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            double t = __shfl_up_sync(0xffffffffu, c, o);
            if (lane >= o) c = t + c;
        }
        const double S = __shfl_sync(0xffffffffu, c, cnt - 1);
        // emission needs random access to (mu, mw, c): stage in shared memory
        s_mu[wib][lane] = mu;
        s_mw[wib][lane] = mw;
        s_c[wib][lane] = c;
        __syncwarp();
        if (lane < cnt) emit_slot(F, v, fi, lane, cnt, s_mu[wib], s_mw[wib], s_c[wib], S);
        if (lane == 0) {
            F.D[v] = S;
            F.Lcnt[v] = cnt;
            F.fcnt[fi] = cnt > 0 ? cnt - 1 : 0;
            if (cnt > 1) atomicAdd((unsigned long long*)&F.ctr[C_NFILL], (unsigned long long)(cnt - 1));
            if (cnt > 1 && F.vseg)
                atomicAdd((unsigned long long*)&F.gctr[3 * F.vseg[v] + GC_NFILL], (unsigned long long)(cnt - 1));
        }
        __syncwarp();
    }
}

// Block helpers -----------------------------------------------------------------
// exclusive block scan of an int flag (one per thread), returns the prefix; *total gets the sum.
__device__ __forceinline__ int32_t block_excl_scan(int32_t x, int32_t* s_warp, int32_t* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    int32_t incl = x;
    for (int o = 1; o < 32; o <<= 1) {
        int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int32_t t = lane < nwarp ? s_warp[lane] : 0;
        int32_t ti = t;
        for (int o = 1; o < 32; o <<= 1) {
            int32_t u = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o) ti += u;
        }
        if (lane < nwarp) s_warp[lane] = ti - t;
        if (lane == 31) s_warp[32] = ti;
    }
    __syncthreads();
    int32_t r = s_warp[wid] + incl - x;
    *total = s_warp[32];
    __syncthreads();
    return r;
}

// Chunked scan of mw[0..cnt) into sc: 32-wide Kogge-Stone chunks, sequential carry.
__device__ void block_chunk_scan(const double* mw, double* sc, int32_t cnt, double* s_carry) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int32_t nch = (cnt + 31) >> 5;
    for (int32_t ch = wid; ch < nch; ch += nwarp) {
        int32_t i = ch * 32 + lane;
        double c = i < cnt ? mw[i] : 0.0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            double t = __shfl_up_sync(0xffffffffu, c, o);
            if (lane >= o) c = t + c;
        }
        if (i < cnt) sc[i] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double carry = 0.0;
        for (int32_t ch = 1; ch < nch; ch++) {
            int32_t last_prev = min(ch * 32, cnt) - 1;  // last element of chunk ch-1
            double prev_local = sc[last_prev];
            carry = (ch == 1) ? prev_local : carry + prev_local;
            s_carry[ch] = carry;
        }
    }
    __syncthreads();
    for (int32_t i = 32 + threadIdx.x; i < cnt; i += blockDim.x) sc[i] = s_carry[i >> 5] + sc[i];
    __syncthreads();
}

// gather live entries of bag[v], sort by (u,w), merge runs.  Returns merged count in mu/mw.
// Arrays hold P slots (P = pow2 >= L).
__device__ int32_t block_gather_merge(const FDev& F, int32_t v, int32_t L, int32_t cap, int32_t* su, double* sw,
                                      int32_t* mu, double* mw, int32_t* s_warp, int32_t* s_cnt) {
    int P = 2;
    while (P < L) P <<= 1;
    if (threadIdx.x == 0) *s_cnt = 0;
    __syncthreads();
    const int64_t s = F.bag_start[v];
    const int32_t len = F.bag_len[v];
    for (int32_t q = threadIdx.x; q < len; q += blockDim.x) {
        int32_t uu = F.pool_u[s + q];
        if (F.level[uu] < 0) {
            int32_t pos = atomicAdd(s_cnt, 1);
            if (pos < L && pos < cap) {
                su[pos] = uu;
                sw[pos] = F.pool_w[s + q];
            } else {
                atomicOr((unsigned long long*)&F.ctr[C_ERR], (unsigned long long)FERR_OVERFLOW);
            }
        }
    }
    __syncthreads();
    for (int32_t i = L + threadIdx.x; i < P; i += blockDim.x) {
        su[i] = INT32_MAX;
        sw[i] = __longlong_as_double(0x7ff0000000000000ll);
    }
    __syncthreads();
    block_bitonic_ent(su, sw, P, EntUW());
    // heads and run sums
    int32_t cnt = 0;
    for (int32_t base = 0; base < L; base += blockDim.x) {
        int32_t i = base + threadIdx.x;
        bool head = i < L && (i == 0 || su[i - 1] != su[i]);
        double sum = 0.0;
        if (head) {
            sum = sw[i];
            for (int32_t j = i + 1; j < L && su[j] == su[i]; j++) sum = sum + sw[j];
        }
        int32_t tot;
        int32_t pos = block_excl_scan(head ? 1 : 0, s_warp, &tot);
        if (head) {
            mu[cnt + pos] = su[i];
            mw[cnt + pos] = sum;
        }
        cnt += tot;
    }
    __syncthreads();
    return cnt;
}

__device__ void block_finish_column(const FDev& F, int32_t v, int64_t fidx, int32_t cnt, int32_t* mu, double* mw,
                                    double* sc, double* s_carry) {
    if (cnt == 0) {
        if (threadIdx.x == 0) {
            F.D[v] = 0.0;
            F.Lcnt[v] = 0;
            if (fidx >= 0) F.fcnt[fidx] = 0;
        }
        __syncthreads();
        return;
    }
    int P = 2;
    while (P < cnt) P <<= 1;
    for (int32_t i = cnt + threadIdx.x; i < P; i += blockDim.x) {
        mu[i] = INT32_MAX;
        mw[i] = __longlong_as_double(0x7ff0000000000000ll);
    }
    __syncthreads();
    block_bitonic_ent(mu, mw, P, EntWU());
    block_chunk_scan(mw, sc, cnt, s_carry);
    const double S = sc[cnt - 1];
    for (int32_t i = threadIdx.x; i < cnt; i += blockDim.x) emit_slot(F, v, fidx, i, cnt, mu, mw, sc, S);
    if (threadIdx.x == 0) {
        F.D[v] = S;
        F.Lcnt[v] = cnt;
        if (fidx >= 0) {
            F.fcnt[fidx] = cnt - 1;
            if (cnt > 1) atomicAdd((unsigned long long*)&F.ctr[C_NFILL], (unsigned long long)(cnt - 1));
            if (cnt > 1 && F.vseg)
                atomicAdd((unsigned long long*)&F.gctr[3 * F.vseg[v] + GC_NFILL], (unsigned long long)(cnt - 1));
        }
    }
    __syncthreads();
}

// Block tier (shared memory) and global tier (scratch slices), one block per vertex.
__global__ void k_elim_block(FDev F, const int32_t* frontier, const int32_t* live_cnt, const int32_t* list,
                             int64_t nlist_idx, int32_t cap, int32_t* g_u, double* g_w) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int32_t s_warp[33];
    __shared__ int32_t s_cnt;
    __shared__ double s_carry_static[BLOCK_TIER_MAX / 32 + 1];
    const int64_t nlist = F.ctr[nlist_idx];
    for (int64_t li = blockIdx.x; li < nlist; li += gridDim.x) {
        const int32_t fi = list[li];
        const int32_t v = frontier[fi];
        const int32_t L = live_cnt[fi];
        int32_t *su, *mu;
        double *sw, *mw, *sc, *s_carry;
        if (g_u) {  // global scratch: 2 int arrays + 3 double arrays of cap, carry after
            int64_t base = (int64_t)blockIdx.x * cap;
            su = g_u + 2 * base;
            mu = su + cap;
            sw = g_w + 4 * base;
            mw = sw + cap;
            sc = mw + cap;
            s_carry = sc + cap;
        } else {
            sw = (double*)smem;
            mw = sw + cap;
            sc = mw + cap;
            su = (int32_t*)(sc + cap);
            mu = su + cap;
            s_carry = s_carry_static;
        }
        int32_t cnt = block_gather_merge(F, v, L, cap, su, sw, mu, mw, s_warp, &s_cnt);
        block_finish_column(F, v, fi, cnt, mu, mw, sc, s_carry);
    }
}

// ---------------------------------------------------------------- release / fill bookkeeping
__global__ void k_release(FDev F, const int32_t* frontier, int32_t* next, int32_t lvl) {
    const int64_t nf = F.ctr[C_REM];
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t fi = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; fi < nf; fi += nw) {
        const int32_t v = frontier[fi];
        const int64_t s = F.bag_start[v];
        const int32_t len = F.bag_len[v];
        for (int32_t q = lane; q < len; q += 32) {
            int32_t u = F.pool_u[s + q];
            if (F.level[u] >= 0) continue;
            int32_t old = atomicSub(&F.count[u], 1);
            if (old == 1) next[atomicAdd((unsigned long long*)&F.ctr[C_NEXT], 1ull)] = u;
        }
        __syncwarp();
        if (lane == 0) F.level[v] = lvl;
    }
}

__global__ void k_fill_incoming(FDev F, int32_t* incoming, int32_t* owners) {
    const int64_t nf = F.ctr[C_REM];
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t fi = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; fi < nf; fi += nw) {
        const int64_t s = F.fstart[fi];
        const int32_t c = F.fcnt[fi];
        for (int32_t q = lane; q < c; q += 32) {
            int32_t a = F.fill_a[s + q], b = F.fill_b[s + q];
            if (atomicAdd(&incoming[a], 1) == 0) owners[atomicAdd((unsigned long long*)&F.ctr[C_OWNERS], 1ull)] = a;
            if (atomicAdd(&incoming[b], 1) == 0) owners[atomicAdd((unsigned long long*)&F.ctr[C_OWNERS], 1ull)] = b;
        }
    }
}

// warp per owner: make room for the incoming fill (relocate, dropping stale entries)
__global__ void k_reserve(FDev F, int32_t* incoming, const int32_t* owners) {
    const int64_t no = F.ctr[C_OWNERS];
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t oi = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; oi < no; oi += nw) {
        const int32_t a = owners[oi];
        const int32_t inc = incoming[a];
        const int32_t len = F.bag_len[a];
        if (len + inc > F.bag_cap[a]) {
            const int64_t s = F.bag_start[a];
            int32_t live = 0;
            for (int32_t q = lane; q < len; q += 32) live += (F.level[F.pool_u[s + q]] < 0) ? 1 : 0;
            for (int o = 16; o > 0; o >>= 1) live += __shfl_xor_sync(0xffffffffu, live, o);
            const int32_t ncap = max(2 * (live + inc), 16);
            int64_t ns = 0;
            if (lane == 0) ns = (int64_t)atomicAdd((unsigned long long*)&F.ctr[C_POOL], (unsigned long long)ncap);
            ns = __shfl_sync(0xffffffffu, ns, 0);
            if (ns + ncap > F.pool_cap) {
                if (lane == 0) atomicOr((unsigned long long*)&F.ctr[C_ERR], (unsigned long long)FERR_POOL);
            } else {
                int32_t out = 0;
                for (int32_t q0 = 0; q0 < len; q0 += 32) {
                    int32_t q = q0 + lane;
                    bool lv = false;
                    int32_t uu = 0;
                    double ww = 0;
                    if (q < len) {
                        uu = F.pool_u[s + q];
                        ww = F.pool_w[s + q];
                        lv = F.level[uu] < 0;
                    }
                    unsigned m = __ballot_sync(0xffffffffu, lv);
                    if (lv) {
                        int32_t p = out + __popc(m & ((1u << lane) - 1u));
                        F.pool_u[ns + p] = uu;
                        F.pool_w[ns + p] = ww;
                    }
                    out += __popc(m);
                }
                __syncwarp();
                if (lane == 0) {
                    F.bag_start[a] = ns;
                    F.bag_len[a] = live;
                    F.bag_cap[a] = ncap;
                }
            }
        }
        __syncwarp();
        if (lane == 0) incoming[a] = 0;
    }
}

__global__ void k_fill_scatter(FDev F) {
    const int64_t nf = F.ctr[C_REM];
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t fi = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; fi < nf; fi += nw) {
        const int64_t s = F.fstart[fi];
        const int32_t c = F.fcnt[fi];
        for (int32_t q = lane; q < c; q += 32) {
            int32_t a = F.fill_a[s + q], b = F.fill_b[s + q];
            double w = F.fill_w[s + q];
            int32_t sa = atomicAdd(&F.bag_len[a], 1);
            if (sa < F.bag_cap[a]) {
                F.pool_u[F.bag_start[a] + sa] = b;
                F.pool_w[F.bag_start[a] + sa] = w;
            } else {
                atomicOr((unsigned long long*)&F.ctr[C_ERR], (unsigned long long)FERR_OVERFLOW);
            }
            int32_t sb = atomicAdd(&F.bag_len[b], 1);
            if (sb < F.bag_cap[b]) {
                F.pool_u[F.bag_start[b] + sb] = a;
                F.pool_w[F.bag_start[b] + sb] = w;
            } else {
                atomicOr((unsigned long long*)&F.ctr[C_ERR], (unsigned long long)FERR_OVERFLOW);
            }
        }
    }
}

// frontier swap bookkeeping: REM <- NEXT, reset per-level cursors
__global__ void k_level_begin(int64_t* ctr, int64_t* gctr, int32_t nseg) {
    ctr[C_REM] = ctr[C_NEXT];
    ctr[C_NEXT] = 0;
    ctr[C_OWNERS] = 0;
    ctr[C_NFILL] = 0;
    for (int32_t g = 0; g < nseg; g++) gctr[3 * g + GC_NFILL] = 0;
}
__global__ void k_level_prep(int64_t* ctr, int64_t* gctr, int32_t nseg) {
    // the upcoming frontier's counts become the live-count kernel's domain
    ctr[C_FCUR] = 0;
    ctr[C_NB] = 0;
    ctr[C_NG] = 0;
    ctr[C_MAXLIVE] = 0;
    for (int32_t g = 0; g < nseg; g++) gctr[3 * g + GC_FCUR] = gctr[3 * g + GC_NFRONT] = 0;
}
__global__ void k_set_ctr(int64_t* ctr, int idx, int64_t v) { ctr[idx] = v; }
// the frontier without the vertices of stopped graphs (order kept)
__global__ void k_drop_stopped(const int32_t* __restrict__ in, int64_t nin, const int32_t* __restrict__ vseg,
                               const int32_t* __restrict__ stopped, int32_t* __restrict__ out, int64_t* cnt) {
    // one block: order-preserving compaction
    __shared__ int32_t s_base;
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();
    for (int64_t b0 = 0; b0 < nin; b0 += blockDim.x) {
        const int64_t i = b0 + threadIdx.x;
        const int keep = i < nin && !stopped[vseg[in[i]]];
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        __shared__ int32_t s_warp[32];
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane == 0) s_warp[w] = __popc(bal);
        __syncthreads();
        int32_t before = 0;
        for (int j = 0; j < w; j++) before += s_warp[j];
        int32_t tot = 0;
        for (int j = 0; j < (int)(blockDim.x >> 5); j++) tot += s_warp[j];
        if (keep) out[s_base + before + __popc(bal & ((1u << lane) - 1u))] = in[i];
        __syncthreads();
        if (threadIdx.x == 0) s_base += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *cnt = s_base;
}
__global__ void k_collect_live_range(int64_t v0, int64_t v1, const int32_t* level, int32_t* rem, int64_t* cnt) {
    for (int64_t v = v0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < v1; v += (int64_t)gridDim.x * blockDim.x)
        if (level[v] < 0) rem[atomicAdd((unsigned long long*)cnt, 1ull)] = (int32_t)v;
}

// ---------------------------------------------------------------- solve schedule
// Thin-level runs (DevFactor::SolveRun) and their step schedules.  Row t of a run depends, in the forward
// solve, on the rows of the same run that its L row reads (lower levels), and in the backward solve on the
// rows its L column reaches (higher levels); its step is one more than the deepest of those (0 if none).
// Steps list the run's storage rows by (step, storage row).  Built on the host from the runs' own rows.
static void build_solve_schedule(Context& C, DevFactor& out, const std::vector<int64_t>& lp, const std::string& tag) {
    const int32_t NL = out.num_levels;
    out.runs.clear();
    for (int32_t l = 0; l < NL;) {
        int32_t r = l;
        while (r < NL && lp[r + 1] - lp[r] <= THIN_ROWS) r++;
        if (r - l >= 2) {
            out.runs.push_back({l, r, 0, 0, 0, 0});
            l = r;
        } else {
            l++;
        }
    }
    if (out.runs.empty()) return;
    // the runs' vertices, row pointers and entries
    struct Host {
        std::vector<int32_t> vert, fidx, bidx;
        std::vector<int64_t> fptr, bptr;
    };
    std::vector<Host> h(out.runs.size());
    auto get = [&](void* dst, const void* src, size_t bytes) {
        if (bytes) SSP_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, C.stream));
    };
    for (size_t u = 0; u < out.runs.size(); u++) {
        const int64_t r0 = lp[out.runs[u].l0], r1 = lp[out.runs[u].l1];
        h[u].vert.resize(r1 - r0);
        h[u].fptr.resize(r1 - r0 + 1);
        h[u].bptr.resize(r1 - r0 + 1);
        get(h[u].vert.data(), out.level_rows + r0, sizeof(int32_t) * (r1 - r0));
        get(h[u].fptr.data(), out.prow_ptr + r0, sizeof(int64_t) * (r1 - r0 + 1));
        get(h[u].bptr.data(), out.pcol_ptr + r0, sizeof(int64_t) * (r1 - r0 + 1));
    }
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    for (auto& x : h) {
        x.fidx.resize(x.fptr.back() - x.fptr.front());
        x.bidx.resize(x.bptr.back() - x.bptr.front());
        get(x.fidx.data(), out.prow_idx + x.fptr.front(), sizeof(int32_t) * x.fidx.size());
        get(x.bidx.data(), out.pcol_idx + x.bptr.front(), sizeof(int32_t) * x.bidx.size());
    }
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    std::vector<int32_t> fsched, bsched, fstep{0}, bstep{0};
    std::vector<int32_t> where(out.n, -1);  // vertex -> local row of the run being scheduled
    // depth of every local row, then a counting sort by depth
    auto schedule = [&](const Host& x, int64_t r0, bool fwd, std::vector<int32_t>& sched, std::vector<int32_t>& step,
                        int32_t& s0, int32_t& s1) {
        const int32_t R = (int32_t)x.vert.size();
        const auto& ptr = fwd ? x.fptr : x.bptr;
        const auto& idx = fwd ? x.fidx : x.bidx;
        std::vector<int32_t> d(R, 0);
        int32_t depth = 0;
        for (int32_t k = 0; k < R; k++) {
            const int32_t t = fwd ? k : R - 1 - k;  // dependencies come first in this order
            int32_t dt = 0;
            for (int64_t e = ptr[t] - ptr[0]; e < ptr[t + 1] - ptr[0]; e++) {
                const int32_t j = where[idx[e]];
                if (j < 0) continue;
                if (fwd ? j >= t : j <= t) throw Error(SSP_ERR_INVALID, "factor: solve schedule out of order");
                dt = std::max(dt, d[j] + 1);
            }
            d[t] = dt;
            depth = std::max(depth, dt + 1);
        }
        std::vector<int32_t> cnt(depth + 1, 0);
        for (int32_t t = 0; t < R; t++) cnt[d[t] + 1]++;
        for (int32_t s = 0; s < depth; s++) cnt[s + 1] += cnt[s];
        const size_t base = sched.size();
        sched.resize(base + R);
        for (int32_t t = 0; t < R; t++) sched[base + cnt[d[t]]++] = (int32_t)(r0 + t);
        s0 = (int32_t)step.size() - 1;
        int32_t acc = (int32_t)base;
        std::vector<int32_t> sz(depth, 0);
        for (int32_t t = 0; t < R; t++) sz[d[t]]++;
        for (int32_t s = 0; s < depth; s++) step.push_back(acc += sz[s]);
        s1 = (int32_t)step.size() - 1;
    };
    for (size_t u = 0; u < out.runs.size(); u++) {
        auto& run = out.runs[u];
        const int64_t r0 = lp[run.l0];
        for (int32_t t = 0; t < (int32_t)h[u].vert.size(); t++) where[h[u].vert[t]] = t;
        schedule(h[u], r0, true, fsched, fstep, run.fs0, run.fs1);
        schedule(h[u], r0, false, bsched, bstep, run.bs0, run.bs1);
        for (int32_t v : h[u].vert) where[v] = -1;
    }
    auto put = [&](const std::vector<int32_t>& v, const char* name) {
        int32_t* d = C.ws.get_t<int32_t>(tag + "_" + name, v.size());
        SSP_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(int32_t) * v.size(), cudaMemcpyHostToDevice, C.stream));
        return d;
    };
    out.fsched = put(fsched, "fsched");
    out.fstep = put(fstep, "fstep");
    out.bsched = put(bsched, "bsched");
    out.bstep = put(bstep, "bstep");
    SSP_CUDA(cudaStreamSynchronize(C.stream));
}

// ---------------------------------------------------------------- dense tail
__global__ void k_collect_live(int64_t n, const int32_t* level, int32_t* rem, int64_t* cnt) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        if (level[v] < 0) rem[atomicAdd((unsigned long long*)cnt, 1ull)] = (int32_t)v;
}

struct KeyVLess {
    const uint64_t* prio;
    __device__ bool operator()(const int32_t& a, const int32_t& b) const {
        uint64_t pa = prio[a], pb = prio[b];
        return pa != pb ? pa < pb : a < b;
    }
};

__global__ void k_sort_rem(int32_t* rem, int32_t T, int32_t P, const uint64_t* prio, int32_t* idx) {
    extern __shared__ int32_t s_keys[];
    for (int i = threadIdx.x; i < P; i += blockDim.x) s_keys[i] = i < T ? rem[i] : -1;
    __syncthreads();
    // -1 sentinels must sort last: compare with sentinel handling
    struct L {
        const uint64_t* prio;
        __device__ bool operator()(const int32_t& a, const int32_t& b) const {
            if (a < 0) return false;
            if (b < 0) return true;
            uint64_t pa = prio[a], pb = prio[b];
            return pa != pb ? pa < pb : a < b;
        }
    } less{prio};
    block_bitonic_kv<false, int32_t, int32_t>(s_keys, (int32_t*)nullptr, P, less);
    for (int i = threadIdx.x; i < T; i += blockDim.x) {
        rem[i] = s_keys[i];
        idx[s_keys[i]] = i;
    }
}

// block per remaining vertex: merged live entries into the dense matrix
__global__ void k_dense_build(FDev F, const int32_t* rem, int32_t T, const int32_t* idx, double* W, int32_t cap,
                              int32_t* g_u, double* g_w, int use_global) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int32_t s_warp[33];
    __shared__ int32_t s_cnt;
    __shared__ int32_t s_live;
    for (int32_t i = blockIdx.x; i < T; i += gridDim.x) {
        const int32_t v = rem[i];
        // live count
        if (threadIdx.x == 0) s_live = 0;
        __syncthreads();
        const int64_t s = F.bag_start[v];
        const int32_t len = F.bag_len[v];
        int32_t c = 0;
        for (int32_t q = threadIdx.x; q < len; q += blockDim.x) c += (F.level[F.pool_u[s + q]] < 0) ? 1 : 0;
        atomicAdd(&s_live, c);
        __syncthreads();
        const int32_t L = s_live;
        int32_t *su, *mu;
        double *sw, *mw;
        if (use_global) {
            int64_t base = (int64_t)blockIdx.x * cap;
            su = g_u + 2 * base;
            mu = su + cap;
            sw = g_w + 4 * base;
            mw = sw + cap;
        } else {
            sw = (double*)smem;
            mw = sw + cap;
            su = (int32_t*)(mw + cap);
            mu = su + cap;
        }
        int32_t cnt = block_gather_merge(F, v, L, cap, su, sw, mu, mw, s_warp, &s_cnt);
        for (int32_t q = threadIdx.x; q < cnt; q += blockDim.x) W[(int64_t)i * T + idx[mu[q]]] = mw[q];
        __syncthreads();
    }
}

// single block: eliminate the T remaining vertices in key order
__global__ void __launch_bounds__(1024) k_dense_elim(FDev F, const int32_t* rem, int32_t T, int32_t Pmax,
                                                     const int32_t* idx, double* W, int64_t Lbase, int32_t lvl0) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int32_t s_warp[33];
    __shared__ double s_carry2[8192 / 32 + 1];
    double* mw = (double*)smem;
    double* sc = mw + Pmax;
    int32_t* mu = (int32_t*)(sc + Pmax);
    int64_t Lpos = Lbase;
    for (int32_t i = 0; i < T; i++) {
        const int32_t v = rem[i];
        const double* row = W + (int64_t)i * T;
        // order-preserving compaction of nonzeros q > i
        int32_t cnt = 0;
        for (int32_t base = i + 1; base < T; base += blockDim.x) {
            int32_t q = base + threadIdx.x;
            double x = q < T ? row[q] : 0.0;
            bool nz = (q < T) && (x != 0.0);
            int32_t tot;
            int32_t pos = block_excl_scan(nz ? 1 : 0, s_warp, &tot);
            if (nz) {
                mu[cnt + pos] = rem[q];
                mw[cnt + pos] = x;
            }
            cnt += tot;
        }
        __syncthreads();
        if (threadIdx.x == 0) F.Lstart[v] = Lpos;
        __syncthreads();
        if (cnt == 0) {
            if (threadIdx.x == 0) {
                F.D[v] = 0.0;
                F.Lcnt[v] = 0;
                F.level[v] = lvl0 + i;
            }
            __syncthreads();
            continue;
        }
        int P = 2;
        while (P < cnt) P <<= 1;
        for (int32_t q = cnt + threadIdx.x; q < P; q += blockDim.x) {
            mu[q] = INT32_MAX;
            mw[q] = __longlong_as_double(0x7ff0000000000000ll);
        }
        __syncthreads();
        block_bitonic_ent(mu, mw, P, EntWU());
        block_chunk_scan(mw, sc, cnt, s_carry2);
        const double S = sc[cnt - 1];
        for (int32_t q = threadIdx.x; q < cnt; q += blockDim.x) {
            F.Lrow[Lpos + q] = mu[q];
            F.Lval[Lpos + q] = -(mw[q] / S);
            if (q + 1 < cnt) {
                const double ci = sc[q];
                const double rem_ = S - ci;
                const double tgt = factor_uniform(F.seed, local_vertex(F.vbase, v), q) * rem_;
                int32_t lo = q + 1, hi = cnt;
                while (lo < hi) {
                    int32_t mid = lo + ((hi - lo) >> 1);
                    if ((sc[mid] - ci) < tgt) lo = mid + 1;
                    else hi = mid;
                }
                const int32_t j = lo < cnt ? lo : cnt - 1;
                const int32_t a = mu[q], b = mu[j];
                const double wf = (mw[q] * rem_) / S;
                const int64_t ia = idx[a], ib = idx[b];
                W[ia * T + ib] = W[ia * T + ib] + wf;
                W[ib * T + ia] = W[ib * T + ia] + wf;
            }
        }
        if (threadIdx.x == 0) {
            F.D[v] = S;
            F.Lcnt[v] = cnt;
            F.level[v] = lvl0 + i;
        }
        Lpos += cnt;
        __syncthreads();
    }
}

// ---------------------------------------------------------------- truncation
// block per remaining vertex: no L entries, D = merged live weights summed in row order
__global__ void k_trunc_diag(FDev F, const int32_t* rem, int32_t T, int32_t lvl, int32_t cap, int32_t* g_u,
                             double* g_w, int use_global) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int32_t s_warp[33];
    __shared__ int32_t s_cnt;
    __shared__ int32_t s_live;
    for (int32_t i = blockIdx.x; i < T; i += gridDim.x) {
        const int32_t v = rem[i];
        if (threadIdx.x == 0) s_live = 0;
        __syncthreads();
        const int64_t s = F.bag_start[v];
        const int32_t len = F.bag_len[v];
        int32_t c = 0;
        for (int32_t q = threadIdx.x; q < len; q += blockDim.x) c += (F.level[F.pool_u[s + q]] < 0) ? 1 : 0;
        atomicAdd(&s_live, c);
        __syncthreads();
        const int32_t L = s_live;
        int32_t *su, *mu;
        double *sw, *mw;
        if (use_global) {
            int64_t base = (int64_t)blockIdx.x * cap;
            su = g_u + 2 * base;
            mu = su + cap;
            sw = g_w + 4 * base;
            mw = sw + cap;
        } else {
            sw = (double*)smem;
            mw = sw + cap;
            su = (int32_t*)(mw + cap);
            mu = su + cap;
        }
        const int32_t cnt = block_gather_merge(F, v, L, cap, su, sw, mu, mw, s_warp, &s_cnt);
        if (threadIdx.x == 0) {
            double d = 0.0;
            for (int32_t q = 0; q < cnt; q++) d = d + mw[q];
            F.D[v] = d;
            F.Lcnt[v] = 0;
            F.Lstart[v] = 0;
        }
        __syncthreads();
    }
}
__global__ void k_set_level(const int32_t* rem, int32_t T, int32_t lvl, int32_t* level) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) level[rem[i]] = lvl;
}

// ---------------------------------------------------------------- post-processing
__global__ void k_copy_cols(int64_t n, const int64_t* Lstart, const int32_t* Lcnt, const int32_t* Lrow,
                            const double* Lval, const int64_t* col_ptr, int32_t* col_idx, double* col_val) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        const int64_t s = Lstart[v], d = col_ptr[v];
        const int32_t c = Lcnt[v];
        for (int32_t q = lane; q < c; q += 32) {
            col_idx[d + q] = Lrow[s + q];
            col_val[d + q] = Lval[s + q];
        }
    }
}

__global__ void k_row_count(int64_t nnz, const int32_t* col_idx, int32_t* rowcnt) {
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&rowcnt[col_idx[p]], 1);
}

__global__ void k_row_scatter(int64_t n, const int64_t* col_ptr, const int32_t* col_idx, const double* col_val,
                              const int64_t* row_ptr, int32_t* cursor, int32_t* row_idx, double* row_val) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        for (int64_t p = col_ptr[v] + lane; p < col_ptr[v + 1]; p += 32) {
            int32_t u = col_idx[p];
            int32_t slot = atomicAdd(&cursor[u], 1);
            row_idx[row_ptr[u] + slot] = (int32_t)v;
            row_val[row_ptr[u] + slot] = col_val[p];
        }
    }
}

__global__ void k_level_count(int64_t n, const int32_t* level, int32_t* lvcnt) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&lvcnt[level[v]], 1);
}
__global__ void k_level_scatter(int64_t n, const int32_t* level, const int64_t* lvptr, int32_t* cursor,
                                int32_t* rows) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        int32_t l = level[v];
        rows[lvptr[l] + atomicAdd(&cursor[l], 1)] = (int32_t)v;
    }
}
__global__ void k_i64_to_i32(int64_t n, const int64_t* a, int32_t* b) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (int32_t)a[i];
}

// ---------------------------------------------------------------- bag pool compaction
// warp per vertex: live bags get 2*live + 8 slots in a fresh pool; eliminated vertices get none
__global__ void k_compact_caps(FDev F, int32_t* newcap) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < F.n; v += nw) {
        int32_t live = 0;
        if (F.level[v] < 0) {
            const int64_t s = F.bag_start[v];
            const int32_t len = F.bag_len[v];
            for (int32_t q = lane; q < len; q += 32) live += (F.level[F.pool_u[s + q]] < 0) ? 1 : 0;
            for (int o = 16; o > 0; o >>= 1) live += __shfl_xor_sync(0xffffffffu, live, o);
        }
        if (lane == 0) newcap[v] = F.level[v] < 0 ? 2 * live + 8 : 0;
    }
}

__global__ void k_compact_copy(FDev F, const int64_t* newstart, const int32_t* newcap, int32_t* nu, double* nw_) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < F.n; v += nw) {
        if (F.level[v] >= 0) continue;
        const int64_t s = F.bag_start[v], d = newstart[v];
        const int32_t len = F.bag_len[v];
        int32_t out = 0;
        for (int32_t q0 = 0; q0 < len; q0 += 32) {
            int32_t q = q0 + lane;
            bool lv = false;
            int32_t uu = 0;
            double ww = 0;
            if (q < len) {
                uu = F.pool_u[s + q];
                ww = F.pool_w[s + q];
                lv = F.level[uu] < 0;
            }
            unsigned m = __ballot_sync(0xffffffffu, lv);
            if (lv) {
                int32_t p = out + __popc(m & ((1u << lane) - 1u));
                nu[d + p] = uu;
                nw_[d + p] = ww;
            }
            out += __popc(m);
        }
        __syncwarp();
        if (lane == 0) {
            F.bag_start[v] = d;
            F.bag_len[v] = out;
            F.bag_cap[v] = newcap[v];
        }
    }
}

// storage-order copies of the row and column forms
__global__ void k_perm_count(int64_t n, const int32_t* perm, const int64_t* ptr, int32_t* cnt) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = perm[i];
        cnt[i] = (int32_t)(ptr[v + 1] - ptr[v]);
    }
}
__global__ void k_perm_copy(int64_t n, const int32_t* perm, const int64_t* ptr, const int32_t* idx, const double* val,
                            const int64_t* pptr, int32_t* pidx, double* pval) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        const int32_t v = perm[i];
        const int64_t s = ptr[v], d = pptr[i], c = ptr[v + 1] - s;
        for (int64_t q = lane; q < c; q += 32) {
            pidx[d + q] = idx[s + q];
            pval[d + q] = val[s + q];
        }
    }
}

// ---------------------------------------------------------------- host driver
// grow a device buffer, keeping its first `keep` bytes
static void* grow_keep(Context& C, const std::string& name, void* old, size_t keep, size_t bytes) {
    (void)old;
    return C.ws.grow(name, keep, bytes, C.stream);
}

void factor_device(Context& C, int64_t n, const int64_t* colptr, const int32_t* rowidx, const double* val,
                   const FactorOptions& opt, DevFactor& out, const std::string& tag) {
    SSP_REQUIRE(n > 0, SSP_ERR_INVALID, "factor: empty matrix");
    SSP_REQUIRE(opt.dense_threshold >= 0 && opt.dense_threshold <= 8192, SSP_ERR_INVALID,
                "factor: dense_threshold must be in [0, 8192]");
    Workspace& W = C.ws;
    auto nm = [&](const char* s) { return tag + "_" + s; };
    FDev F;
    F.n = n;
    F.seed = opt.seed;
    F.vbase = opt.vbase;
    // the dense tail looks at the whole Schur complement and would couple several graphs: a union is
    // eliminated in the sparse phase, and truncated graph by graph (vseg)
    const bool seg_mode = opt.vseg != nullptr;
    const int32_t nseg = seg_mode ? (int32_t)opt.seg_row0.size() - 1 : 0;
    SSP_REQUIRE(!opt.vbase || (opt.dense_threshold == 0 && (opt.max_degree == 0 || seg_mode)), SSP_ERR_INVALID,
                "factor: several graphs at once need dense_threshold = 0 (and the graph of every vertex when "
                "truncating)");
    SSP_REQUIRE(!seg_mode || (nseg >= 1 && opt.seg_row0.front() == 0 && opt.seg_row0.back() == n &&
                              (opt.seg_max_degree.empty() || (int32_t)opt.seg_max_degree.size() == nseg)),
                SSP_ERR_INVALID, "factor: inconsistent graph ranges");
    std::vector<int64_t> g_maxdeg(nseg);
    for (int32_t g = 0; g < nseg; g++) {
        g_maxdeg[g] = opt.seg_max_degree.empty() ? opt.max_degree : opt.seg_max_degree[g];
        SSP_REQUIRE(g_maxdeg[g] >= 0, SSP_ERR_INVALID, "factor: a graph's truncation must be >= 0");
    }
    F.vseg = opt.vseg;
    F.nseg = nseg;
    F.gctr = seg_mode ? W.get_t<int64_t>(nm("gctr"), 3 * (size_t)nseg) : nullptr;
    if (seg_mode) SSP_CUDA(cudaMemsetAsync(F.gctr, 0, sizeof(int64_t) * 3 * nseg, C.stream));
    uint64_t* prio = W.get_t<uint64_t>(nm("prio"), n);
    F.prio = prio;
    F.count = W.get_t<int32_t>(nm("count"), n);
    F.level = W.get_t<int32_t>(nm("level"), n);
    F.bag_start = W.get_t<int64_t>(nm("bag_start"), n + 1);
    F.bag_len = W.get_t<int32_t>(nm("bag_len"), n);
    F.bag_cap = W.get_t<int32_t>(nm("bag_cap"), n + 1);
    F.ctr = W.get_t<int64_t>(nm("ctr"), C_NCTR);
    F.Lstart = W.get_t<int64_t>(nm("Lstart"), n);
    F.Lcnt = W.get_t<int32_t>(nm("Lcnt"), n + 1);
    F.D = W.get_t<double>(nm("D"), n);
    int32_t* deg = W.get_t<int32_t>(nm("deg"), n + 1);
    SSP_CUDA(cudaMemsetAsync(F.ctr, 0, sizeof(int64_t) * C_NCTR, C.stream));
    SSP_CUDA(cudaMemsetAsync(deg, 0, sizeof(int32_t) * (n + 1), C.stream));
    SSP_CUDA(cudaMemsetAsync(F.bag_len, 0, sizeof(int32_t) * n, C.stream));
    SSP_CUDA(cudaMemsetAsync(F.Lcnt, 0, sizeof(int32_t) * (n + 1), C.stream));
    const int T256 = 256;
    k_prio<<<grid_for(n, T256), T256, 0, C.stream>>>(n, opt.seed, prio, opt.vbase);
    k_lower_deg<<<grid_for(n, T256), T256, 0, C.stream>>>(n, colptr, rowidx, val, deg);
    k_bag_caps<<<grid_for(n, T256), T256, 0, C.stream>>>(n, deg, F.bag_cap);
    SSP_CHECK_LAUNCH();
    C.kernels_launched += 3;
    SSP_CUDA(cudaMemsetAsync(F.bag_cap + n, 0, sizeof(int32_t), C.stream));
    int64_t* d_tot = W.get_t<int64_t>(nm("tot"), 2);
    exclusive_scan_i32_to_i64(C, F.bag_cap, F.bag_start, n + 1, d_tot);
    const int64_t pool_init = read_i64(C, d_tot);
    // room for relocations: the live entry count never grows, so 3x the initial layout plus slack
    int64_t pool_cap = pool_init * 4 + 20 * n + 4096;
    F.pool_u = W.get_t<int32_t>(nm("pool_u"), pool_cap);
    F.pool_w = W.get_t<double>(nm("pool_w"), pool_cap);
    F.pool_cap = pool_cap;
    int pool_gen = 0;
    out.frontier_sizes.clear();
    out.compactions = 0;
    out.truncated_rows = 0;
    k_bag_fill<<<grid_for(n, T256), T256, 0, C.stream>>>(n, colptr, rowidx, val, F);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    // pool cursor = pool_init
    SSP_CUDA(cudaMemcpyAsync(F.ctr + C_POOL, d_tot, sizeof(int64_t), cudaMemcpyDeviceToDevice, C.stream));
    int32_t* frontier = W.get_t<int32_t>(nm("frontier"), n);
    int32_t* next = W.get_t<int32_t>(nm("next"), n);
    int32_t* live_cnt = W.get_t<int32_t>(nm("live_cnt"), n);
    int32_t* list_b = W.get_t<int32_t>(nm("list_b"), n);
    int32_t* list_g = W.get_t<int32_t>(nm("list_g"), n);
    int32_t* incoming = W.get_t<int32_t>(nm("incoming"), n);
    int32_t* owners = W.get_t<int32_t>(nm("owners"), n);
    F.fstart = W.get_t<int64_t>(nm("fstart"), n);
    F.fcnt = W.get_t<int32_t>(nm("fcnt"), n);
    SSP_CUDA(cudaMemsetAsync(incoming, 0, sizeof(int32_t) * n, C.stream));
    k_init_count<<<grid_for(n * 32, T256, 148 * 64), T256, 0, C.stream>>>(F, next);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;

    // L pool and fill buffer (grown on demand)
    int64_t Lcap = std::max<int64_t>(pool_init * 2, 1024);
    F.Lrow = W.get_t<int32_t>(nm("Lrow"), Lcap);
    F.Lval = W.get_t<double>(nm("Lval"), Lcap);
    int64_t Fcap = std::max<int64_t>(pool_init, 1024);
    F.fill_a = W.get_t<int32_t>(nm("fill_a"), Fcap);
    F.fill_b = W.get_t<int32_t>(nm("fill_b"), Fcap);
    F.fill_w = W.get_t<double>(nm("fill_w"), Fcap);

    // live counts of the first frontier
    auto live_count = [&](int32_t* fr) {
        k_level_prep<<<1, 1, 0, C.stream>>>(F.ctr, F.gctr, F.nseg);
        k_live_count<<<grid_for(n * 32, T256, 148 * 64), T256, 0, C.stream>>>(F, fr, live_cnt, list_b, list_g);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += 2;
    };
    live_count(next);

    int64_t h[C_NCTR];
    int64_t eliminated = 0;
    int32_t lvl = 0;
    int64_t live_entries = 0;  // live entries of the current Schur complement (both directions)
    {
        SSP_CUDA(cudaMemsetAsync(deg + n, 0, sizeof(int32_t), C.stream));
        int64_t* tmp = W.get_t<int64_t>(nm("degscan"), n + 1);
        exclusive_scan_i32_to_i64(C, deg, tmp, n + 1, d_tot);
        live_entries = read_i64(C, d_tot);
    }
    int64_t prev_fcur = -1;
    bool truncated = false;
    int64_t Lused_prev = 0;
    const size_t blk_smem = (size_t)BLOCK_TIER_MAX * (3 * sizeof(double) + 2 * sizeof(int32_t));
    SSP_CUDA(cudaFuncSetAttribute(k_elim_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)blk_smem));
    // several graphs: each graph's own truncation test, with its own live-entry count (the same accounting
    // as the single-graph test below, restricted to its vertices)
    std::vector<int64_t> g_live(nseg, 0), g_elim(nseg, 0), g_prev(nseg, -1), g_cnt(3 * (size_t)nseg + 1, 0);
    std::vector<int32_t> g_stopped(nseg, 0);
    int32_t* d_stopped = seg_mode ? W.get_t<int32_t>(nm("gstop"), nseg) : nullptr;
    int32_t last_trunc_level = -1;
    if (seg_mode) {
        std::vector<int32_t> hdeg(n);
        SSP_CUDA(cudaMemcpyAsync(hdeg.data(), deg, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
        for (int32_t g = 0; g < nseg; g++)
            for (int64_t v = opt.seg_row0[g]; v < opt.seg_row0[g + 1]; v++) g_live[g] += hdeg[v];
    }
    // graph g's live vertices become its final, diagonal level `at` (k_trunc_diag), as a lone truncation does
    auto truncate_graph = [&](int32_t g, int32_t at) -> int64_t {
        const int64_t v0 = opt.seg_row0[g], v1 = opt.seg_row0[g + 1];
        int32_t* rem = W.get_t<int32_t>(nm("rem"), n + 1);
        SSP_CUDA(cudaMemsetAsync(F.ctr + C_REM, 0, sizeof(int64_t), C.stream));
        k_collect_live_range<<<grid_for(v1 - v0, T256), T256, 0, C.stream>>>(v0, v1, F.level, rem, F.ctr + C_REM);
        SSP_CHECK_LAUNCH();
        const int64_t R = read_i64(C, F.ctr + C_REM);
        if (R == 0) return 0;
        std::vector<int32_t> lens(v1 - v0);
        SSP_CUDA(cudaMemcpyAsync(lens.data(), F.bag_len + v0, sizeof(int32_t) * (v1 - v0), cudaMemcpyDeviceToHost,
                                 C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
        int32_t maxlen = 0;
        for (auto x : lens) maxlen = std::max(maxlen, x);
        int32_t cap = 64;
        while (cap < maxlen) cap <<= 1;
        if (cap <= BLOCK_TIER_MAX) {
            size_t smem = (size_t)cap * (2 * sizeof(double) + 2 * sizeof(int32_t));
            SSP_CUDA(cudaFuncSetAttribute(k_trunc_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_trunc_diag<<<(int)std::min<int64_t>(R, 148 * 8), 256, smem, C.stream>>>(F, rem, (int32_t)R, at, cap,
                                                                                      nullptr, nullptr, 0);
        } else {
            int blocks = 32;
            int32_t* gu = W.get_t<int32_t>(nm("gscr_u"), (size_t)2 * cap * blocks);
            double* gw = W.get_t<double>(nm("gscr_w"), (size_t)4 * cap * blocks);
            k_trunc_diag<<<blocks, 1024, 0, C.stream>>>(F, rem, (int32_t)R, at, cap, gu, gw, 1);
        }
        k_set_level<<<grid_for(R, T256), T256, 0, C.stream>>>(rem, (int32_t)R, at, F.level);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += 3;
        int64_t hh[C_NCTR];
        read_i64s(C, F.ctr, hh, C_NCTR);
        if (hh[C_ERR]) throw Error(SSP_ERR_CAPACITY, "factor: truncation overflow");
        return R;
    };
    while (true) {
        read_i64s(C, F.ctr, h, C_NCTR);
        if (h[C_ERR] & FERR_POOL) throw Error(SSP_ERR_CAPACITY, "factor: bag pool exhausted");
        if (h[C_ERR] & FERR_OVERFLOW) throw Error(SSP_ERR_CAPACITY, "factor: bag overflow");
        if (prev_fcur >= 0) live_entries += 2 * h[C_NFILL] - 2 * prev_fcur;
        int64_t nf = h[C_NEXT];
        if (seg_mode) {
            read_i64s(C, F.gctr, g_cnt.data(), 3 * nseg);
            for (int32_t g = 0; g < nseg; g++)
                if (g_prev[g] >= 0) g_live[g] += 2 * g_cnt[3 * g + GC_NFILL] - 2 * g_prev[g];
        }
        if (nf == 0) break;
        if (seg_mode) {
            std::vector<int32_t> stop;
            for (int32_t g = 0; g < nseg; g++) {
                const int64_t ng = opt.seg_row0[g + 1] - opt.seg_row0[g];
                if (!g_stopped[g] && g_maxdeg[g] > 0 && g_cnt[3 * g + GC_NFRONT] > 0 &&
                    g_live[g] > g_maxdeg[g] * (ng - g_elim[g]))
                    stop.push_back(g);
            }
            if (!stop.empty()) {
                for (int32_t g : stop) {
                    const int64_t R = truncate_graph(g, lvl);
                    g_stopped[g] = 1;
                    eliminated += R;
                    out.truncated_rows += R;
                    last_trunc_level = lvl;
                }
                // the frontier without the stopped graphs, and its reservations made again
                SSP_CUDA(cudaMemcpyAsync(d_stopped, g_stopped.data(), sizeof(int32_t) * nseg, cudaMemcpyHostToDevice,
                                         C.stream));
                k_drop_stopped<<<1, 1024, 0, C.stream>>>(next, nf, F.vseg, d_stopped, frontier, F.ctr + C_NEXT);
                k_set_ctr<<<1, 1, 0, C.stream>>>(F.ctr, C_LCUR, Lused_prev);
                SSP_CHECK_LAUNCH();
                C.kernels_launched += 2;
                std::swap(frontier, next);
                live_count(next);
                read_i64s(C, F.ctr, h, C_NCTR);
                read_i64s(C, F.gctr, g_cnt.data(), 3 * nseg);
                nf = h[C_NEXT];
                if (nf == 0) break;
            }
        }
        if (!seg_mode && opt.max_degree > 0 && live_entries > opt.max_degree * (n - eliminated)) {
            truncated = true;
            break;
        }
        if (eliminated + nf > n || lvl > n)
            throw Error(SSP_ERR_CAPACITY, "factor: frontier accounting inconsistent (eliminated > n)");
        if (opt.dense_threshold > 0 && n - eliminated <= opt.dense_threshold && nf <= DENSE_FRONTIER_MAX) break;
        out.frontier_sizes.push_back(nf);
        // relocations of this level allocate at most 2*(live entries + incoming fill) + 16 per owner
        {
            const int64_t reserve = 2 * (pool_init + 2 * h[C_FCUR]) + 16 * (n - eliminated) + 1024;
            if (h[C_POOL] + reserve > pool_cap) {
                int32_t* newcap = W.get_t<int32_t>(nm("newcap"), n + 1);
                int64_t* newstart = W.get_t<int64_t>(nm("newstart"), n + 1);
                k_compact_caps<<<grid_for(n * 32, T256, 148 * 64), T256, 0, C.stream>>>(F, newcap);
                SSP_CUDA(cudaMemsetAsync(newcap + n, 0, sizeof(int32_t), C.stream));
                exclusive_scan_i32_to_i64(C, newcap, newstart, n + 1, d_tot);
                const int64_t used = read_i64(C, d_tot);
                const int64_t ncap = std::max<int64_t>(pool_cap, used + reserve + used / 2);
                const std::string other = (pool_gen & 1) ? "" : "_b";
                int32_t* nu = W.get_t<int32_t>(nm("pool_u") + other, ncap);
                double* nwp = W.get_t<double>(nm("pool_w") + other, ncap);
                k_compact_copy<<<grid_for(n * 32, T256, 148 * 64), T256, 0, C.stream>>>(F, newstart, newcap, nu, nwp);
                SSP_CHECK_LAUNCH();
                C.kernels_launched += 2;
                F.pool_u = nu;
                F.pool_w = nwp;
                F.pool_cap = pool_cap = ncap;
                SSP_CUDA(cudaMemcpyAsync(F.ctr + C_POOL, d_tot, sizeof(int64_t), cudaMemcpyDeviceToDevice, C.stream));
                pool_gen++;
                out.compactions++;
            }
        }
        // capacities for this level's reservations
        if (h[C_LCUR] > Lcap) {
            int64_t ncap = std::max<int64_t>(h[C_LCUR] + h[C_LCUR] / 2, Lcap * 2);
            F.Lrow = (int32_t*)grow_keep(C, nm("Lrow"), F.Lrow, sizeof(int32_t) * Lused_prev, sizeof(int32_t) * ncap);
            F.Lval = (double*)grow_keep(C, nm("Lval"), F.Lval, sizeof(double) * Lused_prev, sizeof(double) * ncap);
            Lcap = ncap;
        }
        if (h[C_FCUR] > Fcap) {
            Fcap = std::max<int64_t>(h[C_FCUR] + h[C_FCUR] / 2, Fcap * 2);
            F.fill_a = W.get_t<int32_t>(nm("fill_a"), Fcap);
            F.fill_b = W.get_t<int32_t>(nm("fill_b"), Fcap);
            F.fill_w = W.get_t<double>(nm("fill_w"), Fcap);
        }
        Lused_prev = h[C_LCUR];
        prev_fcur = h[C_FCUR];
        for (int32_t g = 0; g < nseg; g++) {
            g_prev[g] = g_cnt[3 * g + GC_FCUR];
            g_elim[g] += g_cnt[3 * g + GC_NFRONT];
        }
        std::swap(frontier, next);
        k_level_begin<<<1, 1, 0, C.stream>>>(F.ctr, F.gctr, F.nseg);  // REM <- NEXT (frontier size), NEXT <- 0
        k_elim_warp<<<grid_for(nf * 32, 128, 148 * 64), 128, 0, C.stream>>>(F, frontier, live_cnt);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += 2;
        if (h[C_NB] > 0) {
            int32_t cap = 64;
            while (cap < std::min<int64_t>(h[C_MAXLIVE], BLOCK_TIER_MAX)) cap <<= 1;
            size_t smem = (size_t)cap * (3 * sizeof(double) + 2 * sizeof(int32_t));
            int blocks = (int)std::min<int64_t>(h[C_NB], 148 * 4);
            k_elim_block<<<blocks, 256, smem, C.stream>>>(F, frontier, live_cnt, list_b, C_NB, cap, nullptr, nullptr);
            SSP_CHECK_LAUNCH();
            C.kernels_launched++;
        }
        if (h[C_NG] > 0) {
            int32_t cap = 64;
            while (cap < h[C_MAXLIVE]) cap <<= 1;
            int blocks = (int)std::min<int64_t>(h[C_NG], 32);
            int32_t* gu = W.get_t<int32_t>(nm("gscr_u"), (size_t)2 * cap * blocks);
            double* gw = W.get_t<double>(nm("gscr_w"), (size_t)4 * cap * blocks);
            k_elim_block<<<blocks, 1024, 0, C.stream>>>(F, frontier, live_cnt, list_g, C_NG, cap, gu, gw);
            SSP_CHECK_LAUNCH();
            C.kernels_launched++;
        }
        const int gw32 = grid_for(nf * 32, T256, 148 * 64);
        k_release<<<gw32, T256, 0, C.stream>>>(F, frontier, next, lvl);
        k_fill_incoming<<<gw32, T256, 0, C.stream>>>(F, incoming, owners);
        k_reserve<<<grid_for(n * 32, T256, 148 * 64), T256, 0, C.stream>>>(F, incoming, owners);
        k_fill_scatter<<<gw32, T256, 0, C.stream>>>(F);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += 4;
        eliminated += nf;
        lvl++;
        live_count(next);
    }
    if (seg_mode && last_trunc_level >= lvl) lvl = last_trunc_level + 1;  // a graph truncated after the last level
    const int32_t sparse_levels = lvl;
    const int64_t T = truncated ? 0 : n - eliminated;
    if (truncated) {
        const int64_t R = n - eliminated;
        int32_t* rem = W.get_t<int32_t>(nm("rem"), R + 1);
        SSP_CUDA(cudaMemsetAsync(F.ctr + C_REM, 0, sizeof(int64_t), C.stream));
        k_collect_live<<<grid_for(n, T256), T256, 0, C.stream>>>(n, F.level, rem, F.ctr + C_REM);
        int32_t maxlen = 0;
        {
            std::vector<int32_t> lens(n);
            SSP_CUDA(cudaMemcpyAsync(lens.data(), F.bag_len, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaStreamSynchronize(C.stream));
            for (auto x : lens) maxlen = std::max(maxlen, x);
        }
        int32_t cap = 64;
        while (cap < maxlen) cap <<= 1;
        if (cap <= BLOCK_TIER_MAX) {
            size_t smem = (size_t)cap * (2 * sizeof(double) + 2 * sizeof(int32_t));
            SSP_CUDA(cudaFuncSetAttribute(k_trunc_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_trunc_diag<<<(int)std::min<int64_t>(R, 148 * 8), 256, smem, C.stream>>>(F, rem, (int32_t)R, lvl, cap,
                                                                                      nullptr, nullptr, 0);
        } else {
            int blocks = 32;
            int32_t* gu = W.get_t<int32_t>(nm("gscr_u"), (size_t)2 * cap * blocks);
            double* gw = W.get_t<double>(nm("gscr_w"), (size_t)4 * cap * blocks);
            k_trunc_diag<<<blocks, 1024, 0, C.stream>>>(F, rem, (int32_t)R, lvl, cap, gu, gw, 1);
        }
        k_set_level<<<grid_for(R, T256), T256, 0, C.stream>>>(rem, (int32_t)R, lvl, F.level);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += 3;
        int64_t hh[C_NCTR];
        read_i64s(C, F.ctr, hh, C_NCTR);
        if (hh[C_ERR]) throw Error(SSP_ERR_CAPACITY, "factor: truncation overflow");
        out.truncated_rows = R;
        lvl++;
    }
    int64_t Lused = Lused_prev;
    // note: Lused_prev covers reservations up to the last processed level
    if (T > 0) {
        // dense tail
        int32_t* rem = W.get_t<int32_t>(nm("rem"), T + 1);
        int32_t* idx = W.get_t<int32_t>(nm("idx"), n);
        SSP_CUDA(cudaMemsetAsync(F.ctr + C_REM, 0, sizeof(int64_t), C.stream));
        k_collect_live<<<grid_for(n, T256), T256, 0, C.stream>>>(n, F.level, rem, F.ctr + C_REM);
        SSP_CHECK_LAUNCH();
        int32_t P = 2;
        while (P < T) P <<= 1;
        SSP_CUDA(cudaFuncSetAttribute(k_sort_rem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(P * sizeof(int32_t))));
        k_sort_rem<<<1, 1024, P * sizeof(int32_t), C.stream>>>(rem, (int32_t)T, P, F.prio, idx);
        SSP_CHECK_LAUNCH();
        double* Wd = W.get_t<double>(nm("W"), (size_t)T * T);
        SSP_CUDA(cudaMemsetAsync(Wd, 0, sizeof(double) * T * T, C.stream));
        // bag sizes bound the build scratch
        int32_t maxlen = 0;
        {
            std::vector<int32_t> lens(n);
            SSP_CUDA(cudaMemcpyAsync(lens.data(), F.bag_len, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaStreamSynchronize(C.stream));
            for (auto x : lens) maxlen = std::max(maxlen, x);
        }
        int32_t cap = 64;
        while (cap < maxlen) cap <<= 1;
        if (cap <= BLOCK_TIER_MAX) {
            size_t smem = (size_t)cap * (2 * sizeof(double) + 2 * sizeof(int32_t));
            SSP_CUDA(cudaFuncSetAttribute(k_dense_build, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_dense_build<<<(int)std::min<int64_t>(T, 148 * 4), 256, smem, C.stream>>>(F, rem, (int32_t)T, idx, Wd,
                                                                                        cap, nullptr, nullptr, 0);
        } else {
            int blocks = 32;
            int32_t* gu = W.get_t<int32_t>(nm("gscr_u"), (size_t)2 * cap * blocks);
            double* gw = W.get_t<double>(nm("gscr_w"), (size_t)4 * cap * blocks);
            k_dense_build<<<blocks, 1024, 0, C.stream>>>(F, rem, (int32_t)T, idx, Wd, cap, gu, gw, 1);
        }
        SSP_CHECK_LAUNCH();
        // L room for the dense phase
        int64_t need = Lused + T * (T - 1) / 2 + 1;
        if (need > Lcap) {
            int64_t ncap = need;
            F.Lrow = (int32_t*)grow_keep(C, nm("Lrow"), F.Lrow, sizeof(int32_t) * Lused, sizeof(int32_t) * ncap);
            F.Lval = (double*)grow_keep(C, nm("Lval"), F.Lval, sizeof(double) * Lused, sizeof(double) * ncap);
            Lcap = ncap;
        }
        // the bitonic sort needs P = pow2 >= T slots per array
        size_t smem = (size_t)P * (2 * sizeof(double) + sizeof(int32_t));
        SSP_CUDA(cudaFuncSetAttribute(k_dense_elim, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_dense_elim<<<1, 1024, smem, C.stream>>>(F, rem, (int32_t)T, P, idx, Wd, Lused, sparse_levels);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += 5;
        Lused += T * (T - 1) / 2;
        int64_t hh[C_NCTR];
        read_i64s(C, F.ctr, hh, C_NCTR);
        if (hh[C_ERR]) throw Error(SSP_ERR_CAPACITY, "factor: dense tail overflow");
    }
    out.n = n;
    out.num_levels = lvl + (int32_t)T;
    out.dense_levels = (int32_t)T;
    // compact columns
    out.col_ptr = W.get_t<int64_t>(nm("col_ptr"), n + 1);
    SSP_CUDA(cudaMemsetAsync(F.Lcnt + n, 0, sizeof(int32_t), C.stream));
    exclusive_scan_i32_to_i64(C, F.Lcnt, out.col_ptr, n + 1, d_tot);
    out.nnz = read_i64(C, d_tot);
    out.col_idx = W.get_t<int32_t>(nm("col_idx"), out.nnz + 1);
    out.col_val = W.get_t<double>(nm("col_val"), out.nnz + 1);
    k_copy_cols<<<grid_for(n * 32, T256, 148 * 64), T256, 0, C.stream>>>(n, F.Lstart, F.Lcnt, F.Lrow, F.Lval,
                                                                        out.col_ptr, out.col_idx, out.col_val);
    SSP_CHECK_LAUNCH();
    // row form
    int32_t* rowcnt = W.get_t<int32_t>(nm("rowcnt"), n + 1);
    int32_t* cursor = W.get_t<int32_t>(nm("rcursor"), n + 1);
    SSP_CUDA(cudaMemsetAsync(rowcnt, 0, sizeof(int32_t) * (n + 1), C.stream));
    SSP_CUDA(cudaMemsetAsync(cursor, 0, sizeof(int32_t) * (n + 1), C.stream));
    k_row_count<<<grid_for(out.nnz, T256), T256, 0, C.stream>>>(out.nnz, out.col_idx, rowcnt);
    SSP_CHECK_LAUNCH();
    out.row_ptr = W.get_t<int64_t>(nm("row_ptr"), n + 1);
    exclusive_scan_i32_to_i64(C, rowcnt, out.row_ptr, n + 1, nullptr);
    out.row_idx = W.get_t<int32_t>(nm("row_idx"), out.nnz + 1);
    out.row_val = W.get_t<double>(nm("row_val"), out.nnz + 1);
    k_row_scatter<<<grid_for(n * 32, T256, 148 * 64), T256, 0, C.stream>>>(n, out.col_ptr, out.col_idx, out.col_val,
                                                                          out.row_ptr, cursor, out.row_idx,
                                                                          out.row_val);
    SSP_CHECK_LAUNCH();
    C.kernels_launched += 4;
    // sort each row by column id (deterministic summation order in the forward solve)
    {
        int64_t* seg_start = out.row_ptr;
        int32_t maxrow = 0;
        std::vector<int32_t> rc(n);
        SSP_CUDA(cudaMemcpyAsync(rc.data(), rowcnt, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
        for (auto x : rc) maxrow = std::max(maxrow, x);
        segsort_pairs_i32_f64(C, out.row_idx, out.row_val, seg_start, rowcnt, n, maxrow);
    }
    out.D = F.D;
    out.level = F.level;
    // level lists
    const int32_t NL = out.num_levels;
    int32_t* lvcnt = W.get_t<int32_t>(nm("lvcnt"), NL + 1);
    int32_t* lvcur = W.get_t<int32_t>(nm("lvcur"), NL + 1);
    SSP_CUDA(cudaMemsetAsync(lvcnt, 0, sizeof(int32_t) * (NL + 1), C.stream));
    SSP_CUDA(cudaMemsetAsync(lvcur, 0, sizeof(int32_t) * (NL + 1), C.stream));
    k_level_count<<<grid_for(n, T256), T256, 0, C.stream>>>(n, F.level, lvcnt);
    SSP_CHECK_LAUNCH();
    int64_t* lvptr = W.get_t<int64_t>(nm("lvptr64"), NL + 1);
    exclusive_scan_i32_to_i64(C, lvcnt, lvptr, NL + 1, nullptr);
    out.level_rows = W.get_t<int32_t>(nm("level_rows"), n);
    k_level_scatter<<<grid_for(n, T256), T256, 0, C.stream>>>(n, F.level, lvptr, lvcur, out.level_rows);
    out.level_ptr_d = W.get_t<int32_t>(nm("level_ptr"), NL + 1);
    k_i64_to_i32<<<grid_for(NL + 1, T256), T256, 0, C.stream>>>(NL + 1, lvptr, out.level_ptr_d);
    SSP_CHECK_LAUNCH();
    C.kernels_launched += 3;
    std::vector<int64_t> lp(NL + 1);
    SSP_CUDA(cudaMemcpyAsync(lp.data(), lvptr, sizeof(int64_t) * (NL + 1), cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    out.level_ptr.assign(NL + 1, 0);
    out.max_level_rows = 0;
    for (int32_t l = 0; l <= NL; l++) out.level_ptr[l] = (int32_t)lp[l];
    for (int32_t l = 0; l < NL; l++) out.max_level_rows = std::max(out.max_level_rows, (int32_t)(lp[l + 1] - lp[l]));
    // storage-order row and column forms + per-level chunk lists
    {
        int32_t* cnt = W.get_t<int32_t>(nm("permcnt"), n + 1);
        auto build = [&](const int64_t* ptr, const int32_t* idx, const double* val, const char* tagp,
                         int64_t** pptr, int32_t** pidx, double** pval, int32_t** chunks,
                         std::vector<int32_t>& chunk_lvl) {
            *pptr = W.get_t<int64_t>(nm(tagp) + "_ptr", n + 1);
            k_perm_count<<<grid_for(n, T256), T256, 0, C.stream>>>(n, out.level_rows, ptr, cnt);
            SSP_CUDA(cudaMemsetAsync(cnt + n, 0, sizeof(int32_t), C.stream));
            exclusive_scan_i32_to_i64(C, cnt, *pptr, n + 1, nullptr);
            *pidx = W.get_t<int32_t>(nm(tagp) + "_idx", out.nnz + 1);
            *pval = W.get_t<double>(nm(tagp) + "_val", out.nnz + 1);
            k_perm_copy<<<grid_for(n * 32, T256, 148 * 64), T256, 0, C.stream>>>(n, out.level_rows, ptr, idx, val,
                                                                                *pptr, *pidx, *pval);
            SSP_CHECK_LAUNCH();
            C.kernels_launched += 2;
            std::vector<int64_t> hp(n + 1);
            SSP_CUDA(cudaMemcpyAsync(hp.data(), *pptr, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaStreamSynchronize(C.stream));
            const int64_t last_nnz = NL > 0 ? hp[lp[NL]] - hp[lp[NL - 1]] : 0;
            if (pptr == &out.prow_ptr) out.last_fwd_nnz = last_nnz;
            else out.last_bwd_nnz = last_nnz;
            std::vector<int32_t> starts;
            chunk_lvl.assign(NL + 1, 0);
            for (int32_t l = 0; l < NL; l++) {
                chunk_lvl[l] = (int32_t)starts.size();
                make_chunks(hp, (int32_t)lp[l], (int32_t)lp[l + 1], starts);
            }
            chunk_lvl[NL] = (int32_t)starts.size();
            starts.push_back((int32_t)n);
            *chunks = W.get_t<int32_t>(nm(tagp) + "_chunks", starts.size());
            SSP_CUDA(cudaMemcpyAsync(*chunks, starts.data(), sizeof(int32_t) * starts.size(), cudaMemcpyHostToDevice,
                                     C.stream));
            SSP_CUDA(cudaStreamSynchronize(C.stream));
        };
        build(out.row_ptr, out.row_idx, out.row_val, "prow", &out.prow_ptr, &out.prow_idx, &out.prow_val,
              &out.fchunk, out.fchunk_lvl);
        build(out.col_ptr, out.col_idx, out.col_val, "pcol", &out.pcol_ptr, &out.pcol_idx, &out.pcol_val,
              &out.bchunk, out.bchunk_lvl);
    }
    build_solve_schedule(C, out, lp, tag);
}

}  // namespace ssp
