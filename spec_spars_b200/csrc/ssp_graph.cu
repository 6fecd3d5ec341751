// ssp_graph.cu -- a2/a3/a5: edges, incidence (implicit) and Laplacian assembly on the device.
//
// Edge order follows the reference exactly: upper-triangle entries (row < col) of the input
// CSC in CSC iteration order, zero values dropped (stream.rs:44-49, sparsifier.rs:357-376).
// B^T (sparsifier.rs:90-114) is never materialised: column e holds -sqrt(w) at v1 and
// +sqrt(w) at v2, which the sketch kernel applies on the fly from the adjacency.
#include "ssp_internal.cuh"

namespace ssp {

enum : int32_t { ERR_RANGE = 1, ERR_ORDER = 2, ERR_WEIGHT = 4 };

// one warp per column: validate and count upper entries
__global__ void k_col_upcount(int64_t n, const int64_t* colptr, const int32_t* rowidx, const double* val,
                              int32_t* upcnt, int32_t* err) {
    int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c = warp; c < n; c += nwarps) {
        int64_t s = colptr[c], e = colptr[c + 1];
        int32_t cnt = 0;
        int32_t bad = (e < s) ? ERR_ORDER : 0;
        for (int64_t p = s + lane; p < e; p += 32) {
            int32_t r = rowidx[p];
            if (r < 0 || r >= n) bad |= ERR_RANGE;
            if (p > s && rowidx[p - 1] >= r) bad |= ERR_ORDER;
            double x = val[p];
            if (r < c && x != 0.0) {
                cnt++;
                if (!(x > 0.0) || !isfinite(x)) bad |= ERR_WEIGHT;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
            bad |= __shfl_xor_sync(0xffffffffu, bad, o);
        }
        if (lane == 0) {
            upcnt[c] = cnt;
            if (bad) atomicOr(err, bad);
        }
    }
}

// one warp per column: emit the upper entries in order (ballot compaction keeps order)
__global__ void k_col_emit(int64_t n, const int64_t* colptr, const int32_t* rowidx, const double* val,
                           const int64_t* eoff, int32_t* v1, int32_t* v2, double* w) {
    int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c = warp; c < n; c += nwarps) {
        int64_t s = colptr[c], e = colptr[c + 1];
        int64_t out = eoff[c];
        for (int64_t p0 = s; p0 < e; p0 += 32) {
            int64_t p = p0 + lane;
            bool take = false;
            int32_t r = 0;
            double x = 0;
            if (p < e) {
                r = rowidx[p];
                x = val[p];
                take = (r < c) && (x != 0.0);
            }
            unsigned mask = __ballot_sync(0xffffffffu, take);
            if (take) {
                int64_t pos = out + __popc(mask & ((1u << lane) - 1u));
                v1[pos] = r;
                v2[pos] = (int32_t)c;
                w[pos] = x;
            }
            out += __popc(mask);
        }
    }
}

__global__ void k_edge_degrees(int64_t m, const int32_t* v1, const int32_t* v2, int32_t* lowcnt, int32_t* highcnt,
                               int32_t* err, int64_t n) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x) {
        int32_t a = v1[e], b = v2[e];
        if (a < 0 || b >= n || a >= b) {
            atomicOr(err, ERR_ORDER);
            continue;
        }
        if (e > 0) {  // CSC order: (v2, v1) strictly increasing
            int32_t pa = v1[e - 1], pb = v2[e - 1];
            if (!(pb < b || (pb == b && pa < a))) atomicOr(err, ERR_ORDER);
        }
        atomicAdd(&lowcnt[b], 1);
        atomicAdd(&highcnt[a], 1);
    }
}

__global__ void k_deg_total(int64_t n, const int32_t* lowcnt, const int32_t* highcnt, int32_t* deg, int32_t* maxdeg) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        int32_t d = lowcnt[v] + highcnt[v];
        deg[v] = d;
        atomicMax(maxdeg, d);
    }
}

// lower part: edge e is the (e - eoff[v2])-th entry of column v2; upper part: atomic cursor, sorted later
__global__ void k_adj_place(int64_t m, const int32_t* v1, const int32_t* v2, const int64_t* eoff,
                            const int64_t* adj_ptr, const int32_t* lowcnt, int32_t* cursor, int32_t* adj_nbr,
                            int32_t* adj_eid) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x) {
        int32_t a = v1[e], b = v2[e];
        int64_t pb = adj_ptr[b] + (e - eoff[b]);
        adj_nbr[pb] = a;
        adj_eid[pb] = (int32_t)e;
        int32_t slot = atomicAdd(&cursor[a], 1);
        int64_t pa = adj_ptr[a] + lowcnt[a] + slot;
        adj_eid[pa] = (int32_t)e;
    }
}

__global__ void k_upper_seg(int64_t n, const int64_t* adj_ptr, const int32_t* lowcnt, const int32_t* highcnt,
                            int64_t* seg_start, int32_t* seg_len) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        seg_start[v] = adj_ptr[v] + lowcnt[v];
        seg_len[v] = highcnt[v];
    }
}

__global__ void k_upper_nbr(int64_t n, const int64_t* adj_ptr, const int32_t* lowcnt, const int32_t* v2,
                            const int32_t* adj_eid, int32_t* adj_nbr) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        for (int64_t p = adj_ptr[v] + lowcnt[v]; p < adj_ptr[v + 1]; p++) adj_nbr[p] = v2[adj_eid[p]];
    }
}

__global__ void k_lap_count(int64_t n, const int32_t* deg, int32_t* lapcnt) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        lapcnt[v] = deg[v] + (deg[v] > 0 ? 1 : 0);
}

// one thread per vertex: diagonal summed in edge order (Triplet::insert, sparsifier.rs:67-68)
// lap_eid[q]: the edge of entry q when its row is the edge's smaller vertex (row < column), else -1; each edge
// is named once, in the column of its larger vertex
__global__ void k_lap_fill(int64_t n, const int64_t* adj_ptr, const int32_t* adj_nbr, const int32_t* adj_eid,
                           const double* w, const int64_t* lap_ptr, int32_t* lap_idx, double* lap_val,
                           int32_t* lap_eid) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        int64_t s = adj_ptr[v], e = adj_ptr[v + 1];
        if (s == e) continue;
        double diag = 0.0;
        for (int64_t p = s; p < e; p++) diag = __dadd_rn(diag, w[adj_eid[p]]);
        int64_t q = lap_ptr[v];
        bool done = false;
        for (int64_t p = s; p < e; p++) {
            int32_t u = adj_nbr[p];
            if (!done && u > v) {
                lap_idx[q] = (int32_t)v;
                lap_eid[q] = -1;
                lap_val[q++] = diag;
                done = true;
            }
            lap_idx[q] = u;
            lap_eid[q] = u < v ? adj_eid[p] : -1;
            lap_val[q++] = -w[adj_eid[p]];
        }
        if (!done) {
            lap_idx[q] = (int32_t)v;
            lap_eid[q] = -1;
            lap_val[q] = diag;
        }
    }
}

static void check_err(Context& C, int32_t* d_err, const char* what) {
    int32_t h = 0;
    SSP_CUDA(cudaMemcpyAsync(&h, d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    if (h & ERR_RANGE) throw Error(SSP_ERR_INVALID, std::string(what) + ": row index out of range");
    if (h & ERR_ORDER)
        throw Error(SSP_ERR_INVALID, std::string(what) + ": indices not strictly increasing (CSC order required)");
    if (h & ERR_WEIGHT)
        throw Error(SSP_ERR_INVALID,
                    std::string(what) + ": edge weights must be finite and positive (upper-triangle entries)");
}

void build_graph_from_edges(Context& C, DevGraph& G, const std::string& tag) {
    const int64_t n = G.n, m = G.m;
    Workspace& W = C.ws;
    int32_t* lowcnt = W.get_t<int32_t>(tag + "_lowcnt", n + 1);
    int32_t* highcnt = W.get_t<int32_t>(tag + "_highcnt", n + 1);
    int32_t* deg = W.get_t<int32_t>(tag + "_deg", n + 1);
    int32_t* cursor = W.get_t<int32_t>(tag + "_cursor", n + 1);
    int32_t* err = W.get_t<int32_t>(tag + "_err", 2);
    SSP_CUDA(cudaMemsetAsync(lowcnt, 0, sizeof(int32_t) * (n + 1), C.stream));
    SSP_CUDA(cudaMemsetAsync(highcnt, 0, sizeof(int32_t) * (n + 1), C.stream));
    SSP_CUDA(cudaMemsetAsync(cursor, 0, sizeof(int32_t) * (n + 1), C.stream));
    SSP_CUDA(cudaMemsetAsync(err, 0, sizeof(int32_t) * 2, C.stream));
    k_edge_degrees<<<grid_for(m, 256), 256, 0, C.stream>>>(m, G.v1, G.v2, lowcnt, highcnt, err, n);
    SSP_CHECK_LAUNCH();
    k_deg_total<<<grid_for(n, 256), 256, 0, C.stream>>>(n, lowcnt, highcnt, deg, err + 1);
    SSP_CHECK_LAUNCH();
    C.kernels_launched += 2;
    check_err(C, err, "edge list");
    int32_t hmax = 0;
    SSP_CUDA(cudaMemcpyAsync(&hmax, err + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    G.max_deg = hmax;

    int64_t* eoff = W.get_t<int64_t>(tag + "_eoff", n + 1);
    exclusive_scan_i32_to_i64(C, lowcnt, eoff, n, nullptr);
    G.adj_ptr = W.get_t<int64_t>(tag + "_adj_ptr", n + 1);
    SSP_CUDA(cudaMemsetAsync(deg + n, 0, sizeof(int32_t), C.stream));
    exclusive_scan_i32_to_i64(C, deg, G.adj_ptr, n + 1, nullptr);  // deg[n] == 0 -> adj_ptr[n] = 2m
    G.adj_nbr = W.get_t<int32_t>(tag + "_adj_nbr", 2 * m + 1);
    G.adj_eid = W.get_t<int32_t>(tag + "_adj_eid", 2 * m + 1);
    k_adj_place<<<grid_for(m, 256), 256, 0, C.stream>>>(m, G.v1, G.v2, eoff, G.adj_ptr, lowcnt, cursor, G.adj_nbr,
                                                         G.adj_eid);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    // upper parts: sort edge ids (edge id order == neighbour order)
    int64_t* seg_start = W.get_t<int64_t>(tag + "_seg_start", n + 1);
    int32_t* seg_len = W.get_t<int32_t>(tag + "_seg_len", n + 1);
    k_upper_seg<<<grid_for(n, 256), 256, 0, C.stream>>>(n, G.adj_ptr, lowcnt, highcnt, seg_start, seg_len);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    segsort_i32(C, G.adj_eid, seg_start, seg_len, n, G.max_deg);
    k_upper_nbr<<<grid_for(n, 256), 256, 0, C.stream>>>(n, G.adj_ptr, lowcnt, G.v2, G.adj_eid, G.adj_nbr);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;

    // Laplacian
    int32_t* lapcnt = W.get_t<int32_t>(tag + "_lapcnt", n + 1);
    k_lap_count<<<grid_for(n, 256), 256, 0, C.stream>>>(n, deg, lapcnt);
    SSP_CHECK_LAUNCH();
    SSP_CUDA(cudaMemsetAsync(lapcnt + n, 0, sizeof(int32_t), C.stream));
    G.lap_ptr = W.get_t<int64_t>(tag + "_lap_ptr", n + 1);
    int64_t* d_tot = W.get_t<int64_t>(tag + "_lap_tot", 1);
    exclusive_scan_i32_to_i64(C, lapcnt, G.lap_ptr, n + 1, d_tot);
    G.lap_nnz = read_i64(C, d_tot);
    G.lap_idx = W.get_t<int32_t>(tag + "_lap_idx", G.lap_nnz + 1);
    G.lap_val = W.get_t<double>(tag + "_lap_val", G.lap_nnz + 1);
    G.lap_eid = W.get_t<int32_t>(tag + "_lap_eid", G.lap_nnz + 1);
    k_lap_fill<<<grid_for(n, 128), 128, 0, C.stream>>>(n, G.adj_ptr, G.adj_nbr, G.adj_eid, G.w, G.lap_ptr,
                                                       G.lap_idx, G.lap_val, G.lap_eid);
    SSP_CHECK_LAUNCH();
    C.kernels_launched += 2;
}

void build_graph_from_csc(Context& C, int64_t n, const int64_t* colptr, const int32_t* rowidx, const double* val,
                          int64_t nnz, DevGraph& G, const std::string& tag) {
    (void)nnz;
    Workspace& W = C.ws;
    G.n = n;
    int32_t* upcnt = W.get_t<int32_t>(tag + "_upcnt", n + 1);
    int32_t* err = W.get_t<int32_t>(tag + "_err", 2);
    SSP_CUDA(cudaMemsetAsync(err, 0, sizeof(int32_t) * 2, C.stream));
    int threads = 256;
    int blocks = grid_for(n * 32, threads, 148 * 64);
    k_col_upcount<<<blocks, threads, 0, C.stream>>>(n, colptr, rowidx, val, upcnt, err);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    check_err(C, err, "input matrix");
    int64_t* eoff = W.get_t<int64_t>(tag + "_eoff_in", n + 1);
    int64_t* d_m = W.get_t<int64_t>(tag + "_m", 1);
    exclusive_scan_i32_to_i64(C, upcnt, eoff, n, d_m);
    G.m = read_i64(C, d_m);
    SSP_REQUIRE(G.m < (int64_t)INT32_MAX, SSP_ERR_INVALID, "more than 2^31-1 edges");
    G.v1 = W.get_t<int32_t>(tag + "_v1", G.m + 1);
    G.v2 = W.get_t<int32_t>(tag + "_v2", G.m + 1);
    G.w = W.get_t<double>(tag + "_w", G.m + 1);
    k_col_emit<<<blocks, threads, 0, C.stream>>>(n, colptr, rowidx, val, eoff, G.v1, G.v2, G.w);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    build_graph_from_edges(C, G, tag);
}

// ---------------------------------------------------------------- Laplacian input
// A Laplacian given as the input (Sparsifier::from_matrix, sparsifier.rs:299-300): the graph is its off-diagonal
// entries negated, in their stored order, zeros kept (edge extraction drops them later, as for any graph).  The
// counts pass checks that the column pointers do not decrease and stay within nnz.
namespace {
__global__ void k_lap_offdiag_count(int64_t n, int64_t nnz, const int64_t* __restrict__ ptr,
                                    const int32_t* __restrict__ idx, int32_t* __restrict__ cnt, int32_t* err) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = ptr[j], e = ptr[j + 1];
        if (s > e || e > nnz || s < 0) {
            atomicOr(err, ERR_ORDER);
            cnt[j] = 0;
            continue;
        }
        int32_t c = 0;
        for (int64_t t = s; t < e; t++) c += idx[t] != (int32_t)j;
        cnt[j] = c;
    }
}
__global__ void k_lap_offdiag_fill(int64_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                   const double* __restrict__ val, const int64_t* __restrict__ optr,
                                   int32_t* __restrict__ oidx, double* __restrict__ oval) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        int64_t o = optr[j];
        for (int64_t t = ptr[j]; t < ptr[j + 1]; t++)
            if (idx[t] != (int32_t)j) {
                oidx[o] = idx[t];
                oval[o] = -val[t];
                o++;
            }
    }
}
}  // namespace

int64_t laplacian_to_graph_device(Context& C, int64_t n, int64_t nnz, const int64_t* ptr, const int32_t* idx,
                                  const double* val, int64_t** gptr, int32_t** gidx, double** gval,
                                  const std::string& tag) {
    Workspace& W = C.ws;
    int64_t ends[2] = {0, 0};
    SSP_CUDA(cudaMemcpyAsync(&ends[0], ptr, sizeof(int64_t), cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaMemcpyAsync(&ends[1], ptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    SSP_REQUIRE(ends[0] == 0 && ends[1] == nnz, SSP_ERR_INVALID, "CSC colptr must start at 0 and end at nnz");
    int32_t* cnt = W.get_t<int32_t>(tag + "_cnt", n + 1);
    int32_t* err = W.get_t<int32_t>(tag + "_err", 1);
    SSP_CUDA(cudaMemsetAsync(err, 0, sizeof(int32_t), C.stream));
    const int blocks = grid_for(n, 256, 148 * 16);
    k_lap_offdiag_count<<<blocks, 256, 0, C.stream>>>(n, nnz, ptr, idx, cnt, err);
    SSP_CHECK_LAUNCH();
    int32_t herr = 0;
    SSP_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int32_t), cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    SSP_REQUIRE(herr == 0, SSP_ERR_INVALID, "CSC colptr must be non-decreasing");
    *gptr = W.get_t<int64_t>(tag + "_ptr", n + 1);
    exclusive_scan_i32_to_i64(C, cnt, *gptr, n, *gptr + n);
    const int64_t gnnz = read_i64(C, *gptr + n);
    *gidx = W.get_t<int32_t>(tag + "_idx", gnnz + 1);
    *gval = W.get_t<double>(tag + "_val", gnnz + 1);
    k_lap_offdiag_fill<<<blocks, 256, 0, C.stream>>>(n, ptr, idx, val, *gptr, *gidx, *gval);
    SSP_CHECK_LAUNCH();
    C.kernels_launched += 2;
    return gnnz;
}

// ---------------------------------------------------------------- streaming update
// Sparsifier::form_laplacian (sparsifier.rs:693-709) adds the Laplacian of the edges inserted since the last
// sparsification to the current one.  Here the sum is formed as a graph: the current Laplacian's
// off-diagonal nonzeros become edges of weight -value, the new batch's entries are added column by column
// (duplicates summed current + new, which is exactly -(L_cur + L_new) off the diagonal), and the Laplacian is
// rebuilt from that graph, its diagonal summed in edge order.
namespace {
__global__ void k_lap_graph_count(int64_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                  const double* __restrict__ val, int32_t* __restrict__ cnt) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        int32_t c = 0;
        for (int64_t t = ptr[j]; t < ptr[j + 1]; t++) c += (idx[t] != (int32_t)j && val[t] != 0.0);
        cnt[j] = c;
    }
}
__global__ void k_lap_graph_fill(int64_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                 const double* __restrict__ val, const int64_t* __restrict__ optr,
                                 int32_t* __restrict__ oidx, double* __restrict__ oval) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        int64_t o = optr[j];
        for (int64_t t = ptr[j]; t < ptr[j + 1]; t++)
            if (idx[t] != (int32_t)j && val[t] != 0.0) {
                oidx[o] = idx[t];
                oval[o] = -val[t];
                o++;
            }
    }
}
// C = A + B column by column; rows are sorted within each column of A and B
__global__ void k_csc_add_count(int64_t n, const int64_t* __restrict__ ap, const int32_t* __restrict__ ai,
                                const int64_t* __restrict__ bp, const int32_t* __restrict__ bi,
                                int32_t* __restrict__ cnt) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        int64_t x = ap[j], y = bp[j];
        const int64_t xe = ap[j + 1], ye = bp[j + 1];
        int32_t c = 0;
        while (x < xe || y < ye) {
            if (y >= ye || (x < xe && ai[x] < bi[y])) x++;
            else if (x >= xe || bi[y] < ai[x]) y++;
            else {
                x++;
                y++;
            }
            c++;
        }
        cnt[j] = c;
    }
}
__global__ void k_csc_add_fill(int64_t n, const int64_t* __restrict__ ap, const int32_t* __restrict__ ai,
                               const double* __restrict__ av, const int64_t* __restrict__ bp,
                               const int32_t* __restrict__ bi, const double* __restrict__ bv,
                               const int64_t* __restrict__ cp, int32_t* __restrict__ ci, double* __restrict__ cv) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        int64_t x = ap[j], y = bp[j], o = cp[j];
        const int64_t xe = ap[j + 1], ye = bp[j + 1];
        while (x < xe || y < ye) {
            if (y >= ye || (x < xe && ai[x] < bi[y])) {
                ci[o] = ai[x];
                cv[o] = av[x];
                x++;
            } else if (x >= xe || bi[y] < ai[x]) {
                ci[o] = bi[y];
                cv[o] = bv[y];
                y++;
            } else {
                ci[o] = ai[x];
                cv[o] = __dadd_rn(av[x], bv[y]);
                x++;
                y++;
            }
            o++;
        }
    }
}
}  // namespace

int64_t laplacian_plus_graph_device(Context& C, int64_t n, const int64_t* lptr, const int32_t* lidx,
                                    const double* lval, const int64_t* bptr, const int32_t* bidx, const double* bval,
                                    int64_t** mptr, int32_t** midx, double** mval) {
    Workspace& W = C.ws;
    int32_t* cnt = W.get_t<int32_t>("u_cnt", n + 1);
    int64_t* gptr = W.get_t<int64_t>("u_gptr", n + 1);
    int64_t* tot = W.get_t<int64_t>("u_tot", 1);
    k_lap_graph_count<<<grid_for(n, 256), 256, 0, C.stream>>>(n, lptr, lidx, lval, cnt);
    SSP_CHECK_LAUNCH();
    SSP_CUDA(cudaMemsetAsync(cnt + n, 0, sizeof(int32_t), C.stream));
    exclusive_scan_i32_to_i64(C, cnt, gptr, n + 1, tot);
    const int64_t gnnz = read_i64(C, tot);
    int32_t* gidx = W.get_t<int32_t>("u_gidx", gnnz + 1);
    double* gval = W.get_t<double>("u_gval", gnnz + 1);
    k_lap_graph_fill<<<grid_for(n, 256), 256, 0, C.stream>>>(n, lptr, lidx, lval, gptr, gidx, gval);
    k_csc_add_count<<<grid_for(n, 256), 256, 0, C.stream>>>(n, gptr, gidx, bptr, bidx, cnt);
    SSP_CHECK_LAUNCH();
    int64_t* cptr = W.get_t<int64_t>("u_mptr", n + 1);
    SSP_CUDA(cudaMemsetAsync(cnt + n, 0, sizeof(int32_t), C.stream));
    exclusive_scan_i32_to_i64(C, cnt, cptr, n + 1, tot);
    const int64_t cnnz = read_i64(C, tot);
    int32_t* cidx = W.get_t<int32_t>("u_midx", cnnz + 1);
    double* cval = W.get_t<double>("u_mval", cnnz + 1);
    k_csc_add_fill<<<grid_for(n, 256), 256, 0, C.stream>>>(n, gptr, gidx, gval, bptr, bidx, bval, cptr, cidx, cval);
    SSP_CHECK_LAUNCH();
    C.kernels_launched += 4;
    *mptr = cptr;
    *midx = cidx;
    *mval = cval;
    return cnnz;
}

}  // namespace ssp
