// ssp_mtxio.cu -- Matrix Market ingest and egest on the device.
//
// read_mtx_device gives the same CSC as the host reader (read_mtx, which restates utils::read_mtx,
// utils.rs:149-154: symmetric storage expanded, duplicates summed in file order, rows sorted):
//   1. the header (banner, comments, size line) is parsed on the host with the host reader's checks;
//   2. the body streams to the device through two pinned staging buffers (read and copy overlap);
//   3. newlines are counted per 4 KB tile and scanned into line starts;
//   4. one thread per line parses "row col [value]" (values through the exact decimal conversion of
//      ssp_decimal.cuh); the rare token it cannot convert exactly is parsed with strtod on the host;
//   5. entries are expanded as the host reader pushes them ((i, j), then (j, i) for an off-diagonal entry
//      of a symmetric file), stably radix-sorted by (column, row), and equal keys summed in push order.
// A body the per-line parser cannot mirror exactly (an entry split over lines, extra tokens, a comment
// after the size line) makes the whole file fall back to the host reader, so both paths always agree.
//
// write_mtx_device writes the host writer's bytes (write_mtx: "coordinate real general", one
// "row col %.17g" line per stored entry in CSC order): values are formatted on the device (format_g17),
// lines are sized, scanned and written into one buffer, and the buffer streams back to the file.
#include <sys/stat.h>

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ssp_decimal.cuh"
#include "ssp_host.h"
#include "ssp_internal.cuh"

namespace ssp {

namespace {
constexpr int NL_THREADS = 256;
constexpr int NL_BYTES = 16;                    // bytes per thread
constexpr int NL_TILE = NL_THREADS * NL_BYTES;  // bytes per block
constexpr size_t STAGE_BYTES = 32u << 20;       // pinned staging buffer (two of them)
constexpr int32_t HOST_FIX_CAP = 1 << 14;       // values converted on the host; beyond, the host reads the file

enum : int32_t { LN_BLANK = 0, LN_ENTRY = 1, LN_FALLBACK = 2 };
enum : int32_t { VAL_OK = 0, VAL_HOST = 1 };
}  // namespace

// ---------------------------------------------------------------- self-checks
// Every kernel below checks its writes against the sizes it was given; a violation records (check id, index)
// in *err (the smallest wins) and skips the access.  The host reads *err after each stage.
__device__ __forceinline__ void check_fail(unsigned long long* err, int id, int64_t i) {
    atomicMin(err, ((unsigned long long)id << 48) | ((unsigned long long)i & ((1ull << 48) - 1)));
}

static void stage_check(Context& C, unsigned long long* err, const char* stage) {
    unsigned long long h = ~0ull;
    SSP_CUDA(cudaMemcpyAsync(&h, err, sizeof h, cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    if (h != ~0ull)
        throw Error(SSP_ERR_INVALID, std::string("mtx ") + stage + ": device check " + std::to_string(h >> 48) +
                                         " failed at index " + std::to_string(h & ((1ull << 48) - 1)));
}

// ---------------------------------------------------------------- line index
__global__ void __launch_bounds__(NL_THREADS) k_nl_count(const char* __restrict__ buf, int64_t size,
                                                         int32_t* __restrict__ cnt) {
    __shared__ int32_t s;
    if (threadIdx.x == 0) s = 0;
    __syncthreads();
    const int64_t b = (int64_t)blockIdx.x * NL_TILE + (int64_t)threadIdx.x * NL_BYTES;
    int32_t c = 0;
    for (int i = 0; i < NL_BYTES; i++)
        if (b + i < size && buf[b + i] == '\n') c++;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(&s, c);
    __syncthreads();
    if (threadIdx.x == 0) cnt[blockIdx.x] = s;
}

// line l starts at 0 (l = 0) or one past the l-th newline; the tile's newlines are ranked in byte order
__global__ void __launch_bounds__(NL_THREADS) k_nl_starts(const char* __restrict__ buf, int64_t size,
                                                          const int64_t* __restrict__ off,
                                                          int64_t* __restrict__ starts, int64_t nlines,
                                                          unsigned long long* __restrict__ err) {
    __shared__ int32_t s_warp[NL_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t b = (int64_t)blockIdx.x * NL_TILE + (int64_t)threadIdx.x * NL_BYTES;
    int32_t c = 0;
    for (int i = 0; i < NL_BYTES; i++)
        if (b + i < size && buf[b + i] == '\n') c++;
    int32_t incl = c;
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    int32_t before = 0;
    for (int w = 0; w < warp; w++) before += s_warp[w];
    int64_t r = off[blockIdx.x] + before + incl - c;  // newlines before this thread's bytes
    for (int i = 0; i < NL_BYTES; i++)
        if (b + i < size && buf[b + i] == '\n') {
            if (1 + r < nlines && r >= 0) starts[1 + r] = b + i + 1;
            else check_fail(err, 1, r);
            r++;
        }
    if (blockIdx.x == 0 && threadIdx.x == 0) starts[0] = 0;
}

// ---------------------------------------------------------------- per-line parse
__device__ __forceinline__ bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

// a non-negative or signed decimal integer token, as %lld reads it (no overflow beyond 18 digits)
__device__ __forceinline__ bool parse_int(const char* p, const char* e, int64_t* out) {
    bool neg = false;
    if (p < e && (*p == '+' || *p == '-')) {
        neg = *p == '-';
        p++;
    }
    if (p >= e || p + 18 < e) return false;
    int64_t v = 0;
    for (; p < e; p++) {
        if (*p < '0' || *p > '9') return false;
        v = v * 10 + (*p - '0');
    }
    *out = neg ? -v : v;
    return true;
}

// kind[l]: blank, entry or fallback; for entries I, J (0-based, unchecked) and the value (or a host flag)
__global__ void k_parse_lines(const char* __restrict__ buf, int64_t size, const int64_t* __restrict__ starts,
                              int64_t nlines, int pattern, int32_t* __restrict__ kind, int64_t* __restrict__ I,
                              int64_t* __restrict__ J, double* __restrict__ V, int32_t* __restrict__ vflag) {
    const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlines) return;
    const char* p = buf + starts[l];
    const char* e = buf + (l + 1 < nlines ? starts[l + 1] - 1 : size);  // excludes the newline
    const char* tok[4];
    const char* tend[4];
    int nt = 0;
    while (p < e) {
        while (p < e && is_space(*p)) p++;
        if (p >= e) break;
        if (nt == 4) {
            nt = 5;
            break;
        }
        tok[nt] = p;
        while (p < e && !is_space(*p)) p++;
        tend[nt++] = p;
    }
    if (nt == 0) {
        kind[l] = LN_BLANK;
        return;
    }
    const int want = pattern ? 2 : 3;
    int64_t i, j;
    if (nt != want || *tok[0] == '%' || !parse_int(tok[0], tend[0], &i) || !parse_int(tok[1], tend[1], &j)) {
        kind[l] = LN_FALLBACK;
        return;
    }
    kind[l] = LN_ENTRY;
    I[l] = i - 1;
    J[l] = j - 1;
    if (pattern) {
        V[l] = 1.0;
        vflag[l] = VAL_OK;
        return;
    }
    double v = 0.0;
    const int r = dec::parse_decimal(tok[2], tend[2], &v);
    V[l] = v;
    vflag[l] = r == dec::PARSE_OK ? VAL_OK : VAL_HOST;
}

// entries in line order: rank[l] = entries before line l (exclusive scan of kind == entry); the first nnz
// entries are kept.  Expanded slot of entry t: t + (off-diagonal symmetric entries before t).
__global__ void k_entry_flags(int64_t nlines, const int32_t* __restrict__ kind, int32_t* __restrict__ isent) {
    const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l < nlines) isent[l] = kind[l] == LN_ENTRY;
}

__global__ void k_entry_gather(int64_t nlines, const int32_t* __restrict__ kind, const int64_t* __restrict__ rank,
                               int64_t nnz, int64_t n, const int64_t* __restrict__ I, const int64_t* __restrict__ J,
                               const double* __restrict__ V, int32_t* __restrict__ ei, int32_t* __restrict__ ej,
                               double* __restrict__ ev, int64_t* __restrict__ eline,
                               unsigned long long* __restrict__ first_bad) {
    const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlines || kind[l] != LN_ENTRY) return;
    const int64_t t = rank[l];
    if (t >= nnz) return;
    const int64_t i = I[l], j = J[l];
    if (i < 0 || j < 0 || i >= n || j >= n) {
        atomicMin(first_bad, (unsigned long long)t);
        return;
    }
    ei[t] = (int32_t)i;
    ej[t] = (int32_t)j;
    ev[t] = V[l];
    eline[t] = l;
}

// the first entry line the parser could not mirror (as an entry rank) and the entries whose value needs the
// host, listed up to cap
__global__ void k_line_checks(int64_t nlines, int64_t nnz, const int32_t* __restrict__ kind,
                              const int64_t* __restrict__ rank, const int32_t* __restrict__ vflag,
                              unsigned long long* __restrict__ first_fallback, int32_t* __restrict__ nfix,
                              int64_t* __restrict__ fix, int32_t cap) {
    const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlines || rank[l] >= nnz) return;
    if (kind[l] == LN_FALLBACK) atomicMin(first_fallback, (unsigned long long)rank[l]);
    if (kind[l] == LN_ENTRY && vflag[l] == VAL_HOST) {
        const int32_t q = atomicAdd(nfix, 1);
        if (q < cap) fix[q] = l;
    }
}

__global__ void k_offdiag(int64_t nnz, const int32_t* __restrict__ ei, const int32_t* __restrict__ ej,
                          int32_t* __restrict__ od) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nnz) od[t] = ei[t] != ej[t];
}

// expanded entries in the host reader's push order, keyed by (column, row)
__global__ void k_expand(int64_t nnz, int symmetric, int rbits, const int32_t* __restrict__ ei,
                         const int32_t* __restrict__ ej, const int64_t* __restrict__ odpos,
                         uint64_t* __restrict__ keys, int32_t* __restrict__ src, int64_t E,
                         unsigned long long* __restrict__ err) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nnz) return;
    const int64_t i = ei[t], j = ej[t];
    const int64_t s = t + (symmetric ? odpos[t] : 0);
    if (s < 0 || s + (symmetric && i != j ? 1 : 0) >= E) {
        check_fail(err, 2, t);
        return;
    }
    keys[s] = ((uint64_t)j << rbits) | (uint64_t)i;
    src[s] = (int32_t)t;
    if (symmetric && i != j) {
        keys[s + 1] = ((uint64_t)i << rbits) | (uint64_t)j;
        src[s + 1] = (int32_t)t;
    }
}

__global__ void k_run_heads(int64_t E, const uint64_t* __restrict__ keys, int32_t* __restrict__ head) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < E) head[s] = s == 0 || keys[s] != keys[s - 1];
}

// one thread per run of equal keys: the sum in push order, the row, and the column count
__global__ void k_run_sum(int64_t E, int rbits, const uint64_t* __restrict__ keys, const int32_t* __restrict__ src,
                          const double* __restrict__ ev, const int32_t* __restrict__ head,
                          const int64_t* __restrict__ upos, int32_t* __restrict__ rowidx, double* __restrict__ val,
                          int32_t* __restrict__ colcnt, int64_t U, int64_t n, unsigned long long* __restrict__ err) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= E || !head[s]) return;
    const uint64_t k = keys[s];
    if (upos[s] < 0 || upos[s] >= U || (int64_t)(k >> rbits) >= n || src[s] < 0) {
        check_fail(err, 3, s);
        return;
    }
    double acc = ev[src[s]];
    for (int64_t q = s + 1; q < E && keys[q] == k; q++) acc += ev[src[q]];
    const int64_t u = upos[s];
    rowidx[u] = (int32_t)(k & ((1ull << rbits) - 1));
    val[u] = acc;
    atomicAdd(&colcnt[k >> rbits], 1);
}

// ---------------------------------------------------------------- header (host)
namespace {
struct MtxHeader {
    bool pattern = false, symmetric = false;
    int64_t n = 0, nnz = 0;
    int64_t body = 0;  // byte offset of the first line after the size line
};

bool lower_is(const char* a, const char* b) {
    for (; *a && *b; a++, b++)
        if (tolower((unsigned char)*a) != *b) return false;
    return *a == 0 && *b == 0;
}

// the host reader's header checks and messages
int read_header(FILE* f, MtxHeader& h, std::string& err) {
    char line[4096];
    if (!fgets(line, sizeof line, f)) {
        err = "empty file";
        return -1;
    }
    char banner[64], object[64], format[64], field[64], sym[64];
    if (sscanf(line, "%63s %63s %63s %63s %63s", banner, object, format, field, sym) != 5 ||
        !lower_is(banner, "%%matrixmarket") || !lower_is(object, "matrix") || !lower_is(format, "coordinate")) {
        err = "not a MatrixMarket coordinate matrix";
        return -1;
    }
    h.pattern = lower_is(field, "pattern");
    if (!h.pattern && !lower_is(field, "real") && !lower_is(field, "integer") && !lower_is(field, "double")) {
        err = std::string("unsupported field ") + field;
        return -1;
    }
    h.symmetric = lower_is(sym, "symmetric");
    if (!h.symmetric && !lower_is(sym, "general")) {
        err = std::string("unsupported symmetry ") + sym;
        return -1;
    }
    long long nr = 0, nc = 0, nnz = 0;
    bool got = false;
    while (fgets(line, sizeof line, f)) {
        if (line[0] == '%') continue;
        if (sscanf(line, "%lld %lld %lld", &nr, &nc, &nnz) == 3) {
            got = true;
            break;
        }
        err = "bad size line";
        return -1;
    }
    if (!got || nr <= 0 || nr != nc || nnz < 0) {
        err = "matrix must be square";
        return -1;
    }
    if (strlen(line) == sizeof line - 1 && line[sizeof line - 2] != '\n') {
        err = "size line too long";
        return -1;
    }
    h.n = nr;
    h.nnz = nnz;
    h.body = ftell(f);
    return 0;
}

struct Pinned {
    void* p = nullptr;
    explicit Pinned(size_t bytes) {
        if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            throw Error(SSP_ERR_NOMEM, "pinned host allocation failed");
        }
    }
    ~Pinned() {
        if (p) cudaFreeHost(p);
    }
};

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) fclose(f);
    }
};
}  // namespace

// the rest of an open file (size bytes) into dbuf: fread into one pinned buffer while the other copies
static void upload_body(Context& C, FILE* f, int64_t size, char* dbuf, const char* path) {
    if (size <= 0) return;
    Pinned stage(2 * STAGE_BYTES);
    cudaEvent_t done[2];
    SSP_CUDA(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming));
    SSP_CUDA(cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming));
    int64_t at = 0;
    int slot = 0;
    bool pending[2] = {false, false};
    try {
        while (at < size) {
            char* hb = (char*)stage.p + (size_t)slot * STAGE_BYTES;
            if (pending[slot]) SSP_CUDA(cudaEventSynchronize(done[slot]));
            const size_t want = (size_t)std::min<int64_t>(STAGE_BYTES, size - at);
            const size_t got = fread(hb, 1, want, f);
            if (got != want) throw Error(SSP_ERR_IO, std::string("short read of ") + path);
            SSP_CUDA(cudaMemcpyAsync(dbuf + at, hb, got, cudaMemcpyHostToDevice, C.stream));
            SSP_CUDA(cudaEventRecord(done[slot], C.stream));
            pending[slot] = true;
            at += (int64_t)got;
            slot ^= 1;
        }
        SSP_CUDA(cudaStreamSynchronize(C.stream));
    } catch (...) {
        cudaStreamSynchronize(C.stream);
        cudaEventDestroy(done[0]);
        cudaEventDestroy(done[1]);
        throw;
    }
    cudaEventDestroy(done[0]);
    cudaEventDestroy(done[1]);
}

// line starts of a device text buffer (workspace tag_lstart); returns the line count (the last may be empty)
static int64_t line_index(Context& C, const char* dbuf, int64_t size, const std::string& tag,
                          unsigned long long* derr, int64_t** starts_out) {
    Workspace& W = C.ws;
    auto nm = [&](const char* s) { return tag + "_" + s; };
    const int64_t tiles = std::max<int64_t>(1, ceil_div<int64_t>(size, NL_TILE));
    int32_t* tcnt = W.get_t<int32_t>(nm("nlcnt"), tiles);
    int64_t* toff = W.get_t<int64_t>(nm("nloff"), tiles + 1);
    k_nl_count<<<(unsigned)tiles, NL_THREADS, 0, C.stream>>>(dbuf, size, tcnt);
    SSP_CHECK_LAUNCH();
    exclusive_scan_i32_to_i64(C, tcnt, toff, tiles, toff + tiles);
    const int64_t newlines = read_i64(C, toff + tiles);
    const int64_t nlines = newlines + 1;
    int64_t* starts = W.get_t<int64_t>(nm("lstart"), nlines);
    k_nl_starts<<<(unsigned)tiles, NL_THREADS, 0, C.stream>>>(dbuf, size, toff, starts, nlines, derr);
    SSP_CHECK_LAUNCH();
    C.kernels_launched += 2;
    stage_check(C, derr, "line index");
    *starts_out = starts;
    return nlines;
}

// result: device CSC in workspace buffers tag_{colptr,rowidx,val}; returns false when the file needs the host
// reader (the caller then runs it)
bool read_mtx_device(Context& C, const char* path, int64_t* n_out, int64_t* nnz_out, int64_t** colptr,
                     int32_t** rowidx, double** val, const std::string& tag) {
    File F;
    F.f = fopen(path, "rb");
    if (!F.f) throw Error(SSP_ERR_IO, std::string("cannot open ") + path);
    MtxHeader h;
    std::string err;
    if (read_header(F.f, h, err) != 0) throw Error(SSP_ERR_IO, err);
    if (h.n >= (1ll << 31)) return false;
    struct stat st;
    if (fstat(fileno(F.f), &st) != 0) throw Error(SSP_ERR_IO, std::string("cannot stat ") + path);
    const int64_t size = (int64_t)st.st_size - h.body;
    Workspace& W = C.ws;
    auto nm = [&](const char* s) { return tag + "_" + s; };
    unsigned long long* derr = W.get_t<unsigned long long>(nm("err"), 1);
    SSP_CUDA(cudaMemsetAsync(derr, 0xff, sizeof(unsigned long long), C.stream));
    char* dbuf = W.get_t<char>(nm("text"), (size_t)std::max<int64_t>(size, 1));
    upload_body(C, F.f, size, dbuf, path);
    int64_t* starts = nullptr;
    const int64_t nlines = line_index(C, dbuf, size, tag, derr, &starts);
    // parse
    int32_t* kind = W.get_t<int32_t>(nm("kind"), nlines);
    int64_t* I = W.get_t<int64_t>(nm("li"), nlines);
    int64_t* J = W.get_t<int64_t>(nm("lj"), nlines);
    double* V = W.get_t<double>(nm("lv"), nlines);
    int32_t* vflag = W.get_t<int32_t>(nm("lvf"), nlines);
    const unsigned lb = (unsigned)ceil_div<int64_t>(nlines, 256);
    k_parse_lines<<<lb, 256, 0, C.stream>>>(dbuf, size, starts, nlines, h.pattern ? 1 : 0, kind, I, J, V, vflag);
    SSP_CHECK_LAUNCH();
    stage_check(C, derr, "line parse");
    // entries: rank of every line among the entry lines
    int32_t* isent = W.get_t<int32_t>(nm("isent"), nlines);
    int64_t* rank = W.get_t<int64_t>(nm("rank"), nlines + 1);
    k_entry_flags<<<lb, 256, 0, C.stream>>>(nlines, kind, isent);
    SSP_CHECK_LAUNCH();
    exclusive_scan_i32_to_i64(C, isent, rank, nlines, rank + nlines);
    C.kernels_launched += 2;
    // lines the per-line parser cannot mirror: fall back to the host reader for the whole file, unless they
    // come after the nnz-th entry (the host reader never looks there); values for the host's strtod
    const int64_t nentries = read_i64(C, rank + nlines);
    int64_t* fix = W.get_t<int64_t>(nm("fix"), HOST_FIX_CAP);
    unsigned long long* flags = W.get_t<unsigned long long>(nm("flags"), 2);
    SSP_CUDA(cudaMemsetAsync(flags, 0xff, sizeof(unsigned long long), C.stream));
    SSP_CUDA(cudaMemsetAsync(flags + 1, 0, sizeof(unsigned long long), C.stream));
    k_line_checks<<<lb, 256, 0, C.stream>>>(nlines, h.nnz, kind, rank, vflag, flags, (int32_t*)(flags + 1), fix,
                                            HOST_FIX_CAP);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    unsigned long long hflags[2];
    SSP_CUDA(cudaMemcpyAsync(hflags, flags, sizeof hflags, cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    const int32_t nfix = (int32_t)(hflags[1] & 0xffffffffu);
    if (hflags[0] != ~0ull || nfix > HOST_FIX_CAP) return false;
    // any malformed entry: the host reader runs and reports it exactly as it would
    if (nentries < h.nnz || h.nnz >= (1ll << 31) - 1) return false;
    const int64_t nnz = h.nnz;
    int32_t* ei = W.get_t<int32_t>(nm("ei"), nnz + 1);
    int32_t* ej = W.get_t<int32_t>(nm("ej"), nnz + 1);
    double* ev = W.get_t<double>(nm("ev"), nnz + 1);
    int64_t* eline = W.get_t<int64_t>(nm("eline"), nnz + 1);
    unsigned long long* bad = W.get_t<unsigned long long>(nm("bad"), 1);
    SSP_CUDA(cudaMemsetAsync(bad, 0xff, sizeof(unsigned long long), C.stream));
    k_entry_gather<<<lb, 256, 0, C.stream>>>(nlines, kind, rank, nnz, h.n, I, J, V, ei, ej, ev, eline, bad);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    {
        unsigned long long hb = 0;
        SSP_CUDA(cudaMemcpyAsync(&hb, bad, sizeof hb, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
        if (hb != ~0ull) return false;
    }
    // values the device could not convert exactly: strtod on the host, from the lines' own bytes
    if (nfix > 0) {
        std::vector<int64_t> lines(nfix), hs(1), he(1), hr(1);
        SSP_CUDA(cudaMemcpyAsync(lines.data(), fix, sizeof(int64_t) * nfix, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
        for (int64_t l : lines) {
            SSP_CUDA(cudaMemcpyAsync(hs.data(), starts + l, sizeof(int64_t), cudaMemcpyDeviceToHost, C.stream));
            if (l + 1 < nlines)
                SSP_CUDA(cudaMemcpyAsync(he.data(), starts + l + 1, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                         C.stream));
            else
                he[0] = size;
            SSP_CUDA(cudaMemcpyAsync(hr.data(), rank + l, sizeof(int64_t), cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaStreamSynchronize(C.stream));
            std::string text((size_t)(he[0] - hs[0]), '\0');
            SSP_CUDA(cudaMemcpyAsync(&text[0], dbuf + hs[0], text.size(), cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaStreamSynchronize(C.stream));
            long long a, c;
            double x = 0.0;
            if (sscanf(text.c_str(), "%lld %lld %lf", &a, &c, &x) != 3) return false;
            SSP_CUDA(cudaMemcpyAsync(ev + hr[0], &x, sizeof(double), cudaMemcpyHostToDevice, C.stream));
            SSP_CUDA(cudaStreamSynchronize(C.stream));
        }
    }
    // expand, sort by (column, row) keeping push order, sum equal keys
    int64_t E = nnz;
    int64_t* odpos = nullptr;
    if (h.symmetric && nnz > 0) {
        int32_t* od = W.get_t<int32_t>(nm("od"), nnz);
        odpos = W.get_t<int64_t>(nm("odpos"), nnz + 1);
        k_offdiag<<<(unsigned)ceil_div<int64_t>(nnz, 256), 256, 0, C.stream>>>(nnz, ei, ej, od);
        SSP_CHECK_LAUNCH();
        exclusive_scan_i32_to_i64(C, od, odpos, nnz, odpos + nnz);
        E = nnz + read_i64(C, odpos + nnz);
        C.kernels_launched++;
    }
    int rbits = 1;
    while ((1ll << rbits) < h.n) rbits++;
    uint64_t* keys = W.get_t<uint64_t>(nm("keys"), E + 1);
    int32_t* src = W.get_t<int32_t>(nm("src"), E + 1);
    *colptr = W.get_t<int64_t>(nm("colptr"), h.n + 1);
    int32_t* colcnt = W.get_t<int32_t>(nm("colcnt"), h.n + 1);
    SSP_CUDA(cudaMemsetAsync(colcnt, 0, sizeof(int32_t) * (h.n + 1), C.stream));
    int64_t U = 0;
    if (E > 0) {
        k_expand<<<(unsigned)ceil_div<int64_t>(nnz, 256), 256, 0, C.stream>>>(nnz, h.symmetric ? 1 : 0, rbits, ei,
                                                                               ej, odpos, keys, src, E, derr);
        SSP_CHECK_LAUNCH();
        C.kernels_launched++;
        stage_check(C, derr, "expand");
        uint64_t* tk = W.get_t<uint64_t>(nm("tkeys"), E);
        int32_t* ts = W.get_t<int32_t>(nm("tsrc"), E);
        radix_sort_u64(C, keys, src, E, 2 * rbits, tk, ts, derr);
        stage_check(C, derr, "sort");
        int32_t* head = W.get_t<int32_t>(nm("head"), E);
        int64_t* upos = W.get_t<int64_t>(nm("upos"), E + 1);
        const unsigned eb = (unsigned)ceil_div<int64_t>(E, 256);
        k_run_heads<<<eb, 256, 0, C.stream>>>(E, keys, head);
        SSP_CHECK_LAUNCH();
        exclusive_scan_i32_to_i64(C, head, upos, E, upos + E);
        U = read_i64(C, upos + E);
        *rowidx = W.get_t<int32_t>(nm("rowidx"), U + 1);
        *val = W.get_t<double>(nm("val"), U + 1);
        k_run_sum<<<eb, 256, 0, C.stream>>>(E, rbits, keys, src, ev, head, upos, *rowidx, *val, colcnt, U, h.n, derr);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += 2;
        stage_check(C, derr, "duplicate sums");
    } else {
        *rowidx = W.get_t<int32_t>(nm("rowidx"), 1);
        *val = W.get_t<double>(nm("val"), 1);
    }
    exclusive_scan_i32_to_i64(C, colcnt, *colptr, h.n, *colptr + h.n);
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    *n_out = h.n;
    *nnz_out = U;
    return true;
}

// ---------------------------------------------------------------- egest
namespace {
constexpr int VSLOT = 32;  // bytes per formatted value
}

__device__ __forceinline__ int dec_len(int64_t x) {
    int n = 1;
    while (x >= 10) {
        x /= 10;
        n++;
    }
    return n;
}

__global__ void k_fmt_values(int64_t nnz, const double* __restrict__ val, char* __restrict__ vtxt,
                             int32_t* __restrict__ vlen, unsigned long long* __restrict__ err) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nnz) return;
    char t[VSLOT];
    const int len = dec::format_g17(val[p], t);
    if (len > VSLOT) {
        check_fail(err, 4, p);
        vlen[p] = -1;
        return;
    }
    for (int i = 0; i < len; i++) vtxt[p * VSLOT + i] = t[i];
    vlen[p] = len;
}

__global__ void k_fmt_misses(int64_t nnz, const int32_t* __restrict__ vlen, int32_t* __restrict__ n,
                             int64_t* __restrict__ list, int32_t cap) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < nnz && vlen[p] < 0) {
        const int32_t q = atomicAdd(n, 1);
        if (q < cap) list[q] = p;
    }
}

__global__ void k_col_of(int64_t n, int64_t nnz, const int64_t* __restrict__ colptr, int32_t* __restrict__ col,
                         unsigned long long* __restrict__ err) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int64_t a = colptr[c], b = colptr[c + 1];
    if (a < 0 || b < a || b > nnz) {
        check_fail(err, 5, c);
        return;
    }
    for (int64_t p = a; p < b; p++) col[p] = (int32_t)c;
}

__global__ void k_line_len(int64_t nnz, const int32_t* __restrict__ rowidx, const int32_t* __restrict__ col,
                           const int32_t* __restrict__ vlen, int32_t* __restrict__ llen,
                           unsigned long long* __restrict__ err) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nnz) return;
    if (vlen[p] < 0 || vlen[p] > VSLOT || rowidx[p] < 0 || col[p] < 0) {
        check_fail(err, 6, p);
        llen[p] = 0;
        return;
    }
    llen[p] = dec_len((int64_t)rowidx[p] + 1) + 1 + dec_len((int64_t)col[p] + 1) + 1 + vlen[p] + 1;
}

__device__ __forceinline__ char* put_int(char* o, int64_t x) {
    const int n = dec_len(x);
    for (int i = n - 1; i >= 0; i--) {
        o[i] = (char)('0' + x % 10);
        x /= 10;
    }
    return o + n;
}

__global__ void k_line_write(int64_t nnz, const int32_t* __restrict__ rowidx, const int32_t* __restrict__ col,
                             const char* __restrict__ vtxt, const int32_t* __restrict__ vlen,
                             const int32_t* __restrict__ llen, const int64_t* __restrict__ loff, char* __restrict__ out,
                             int64_t bytes, unsigned long long* __restrict__ err) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nnz) return;
    if (llen[p] <= 0 || loff[p] < 0 || loff[p] + llen[p] > bytes) {
        check_fail(err, 7, p);
        return;
    }
    char* o = out + loff[p];
    o = put_int(o, (int64_t)rowidx[p] + 1);
    *o++ = ' ';
    o = put_int(o, (int64_t)col[p] + 1);
    *o++ = ' ';
    const char* v = vtxt + p * VSLOT;
    for (int i = 0; i < vlen[p]; i++) *o++ = v[i];
    *o = '\n';
}

// the host writer's bytes; colptr/rowidx/val are device arrays
void write_mtx_device(Context& C, const char* path, int64_t n, const int64_t* colptr, const int32_t* rowidx,
                      const double* val, const std::string& tag) {
    Workspace& W = C.ws;
    auto nm = [&](const char* s) { return tag + "_" + s; };
    const int64_t nnz = read_i64(C, colptr + n);
    unsigned long long* derr = W.get_t<unsigned long long>(nm("err"), 1);
    SSP_CUDA(cudaMemsetAsync(derr, 0xff, sizeof(unsigned long long), C.stream));
    File F;
    F.f = fopen(path, "wb");
    if (!F.f) throw Error(SSP_ERR_IO, std::string("cannot open ") + path + " for writing");
    fprintf(F.f, "%%%%MatrixMarket matrix coordinate real general\n");
    fprintf(F.f, "%lld %lld %lld\n", (long long)n, (long long)n, (long long)nnz);
    if (nnz > 0) {
        char* vtxt = W.get_t<char>(nm("vtxt"), (size_t)nnz * VSLOT);
        int32_t* vlen = W.get_t<int32_t>(nm("vlen"), nnz);
        int32_t* col = W.get_t<int32_t>(nm("col"), nnz);
        int32_t* llen = W.get_t<int32_t>(nm("llen"), nnz);
        int64_t* loff = W.get_t<int64_t>(nm("loff"), nnz + 1);
        const unsigned eb = (unsigned)ceil_div<int64_t>(nnz, 256);
        k_fmt_values<<<eb, 256, 0, C.stream>>>(nnz, val, vtxt, vlen, derr);
        k_col_of<<<(unsigned)ceil_div<int64_t>(n, 256), 256, 0, C.stream>>>(n, nnz, colptr, col, derr);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += 2;
        stage_check(C, derr, "format values");
        // values outside the device formatter's range: snprintf on the host
        {
            int32_t* nmiss = W.get_t<int32_t>(nm("nmiss"), 1);
            int64_t* miss = W.get_t<int64_t>(nm("miss"), HOST_FIX_CAP);
            SSP_CUDA(cudaMemsetAsync(nmiss, 0, sizeof(int32_t), C.stream));
            k_fmt_misses<<<eb, 256, 0, C.stream>>>(nnz, vlen, nmiss, miss, HOST_FIX_CAP);
            SSP_CHECK_LAUNCH();
            C.kernels_launched++;
            int32_t hm = 0;
            SSP_CUDA(cudaMemcpyAsync(&hm, nmiss, sizeof hm, cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaStreamSynchronize(C.stream));
            std::vector<int64_t> list;
            if (hm > HOST_FIX_CAP) {  // many: look at every value
                std::vector<int32_t> hl(nnz);
                SSP_CUDA(cudaMemcpyAsync(hl.data(), vlen, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, C.stream));
                SSP_CUDA(cudaStreamSynchronize(C.stream));
                for (int64_t p = 0; p < nnz; p++)
                    if (hl[p] < 0) list.push_back(p);
            } else if (hm > 0) {
                list.resize(hm);
                SSP_CUDA(cudaMemcpyAsync(list.data(), miss, sizeof(int64_t) * hm, cudaMemcpyDeviceToHost, C.stream));
                SSP_CUDA(cudaStreamSynchronize(C.stream));
            }
            for (int64_t p : list) {
                double x = 0.0;
                SSP_CUDA(cudaMemcpyAsync(&x, val + p, sizeof x, cudaMemcpyDeviceToHost, C.stream));
                SSP_CUDA(cudaStreamSynchronize(C.stream));
                char t[64];
                const int len = snprintf(t, sizeof t, "%.17g", x);
                if (len <= 0 || len > VSLOT) throw Error(SSP_ERR_IO, "value too long to format");
                const int32_t l32 = len;
                SSP_CUDA(cudaMemcpyAsync(vtxt + p * VSLOT, t, len, cudaMemcpyHostToDevice, C.stream));
                SSP_CUDA(cudaMemcpyAsync(vlen + p, &l32, sizeof l32, cudaMemcpyHostToDevice, C.stream));
                SSP_CUDA(cudaStreamSynchronize(C.stream));
            }
        }
        k_line_len<<<eb, 256, 0, C.stream>>>(nnz, rowidx, col, vlen, llen, derr);
        SSP_CHECK_LAUNCH();
        stage_check(C, derr, "line lengths");
        exclusive_scan_i32_to_i64(C, llen, loff, nnz, loff + nnz);
        const int64_t bytes = read_i64(C, loff + nnz);
        char* out = W.get_t<char>(nm("out"), (size_t)bytes);
        k_line_write<<<eb, 256, 0, C.stream>>>(nnz, rowidx, col, vtxt, vlen, llen, loff, out, bytes, derr);
        SSP_CHECK_LAUNCH();
        C.kernels_launched += 2;
        stage_check(C, derr, "line write");
        // stream back through two pinned buffers
        Pinned stage(2 * STAGE_BYTES);
        cudaEvent_t done[2];
        SSP_CUDA(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming));
        SSP_CUDA(cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming));
        try {
            int64_t at = 0;
            int slot = 0;
            size_t len[2] = {0, 0};
            bool pending[2] = {false, false};
            auto flush = [&](int s) {
                SSP_CUDA(cudaEventSynchronize(done[s]));
                if (fwrite((char*)stage.p + (size_t)s * STAGE_BYTES, 1, len[s], F.f) != len[s])
                    throw Error(SSP_ERR_IO, "write failed");
                pending[s] = false;
            };
            while (at < bytes) {
                if (pending[slot]) flush(slot);
                len[slot] = (size_t)std::min<int64_t>(STAGE_BYTES, bytes - at);
                SSP_CUDA(cudaMemcpyAsync((char*)stage.p + (size_t)slot * STAGE_BYTES, out + at, len[slot],
                                         cudaMemcpyDeviceToHost, C.stream));
                SSP_CUDA(cudaEventRecord(done[slot], C.stream));
                pending[slot] = true;
                at += (int64_t)len[slot];
                slot ^= 1;
            }
            // the older of the two slots first
            if (pending[slot]) flush(slot);
            if (pending[slot ^ 1]) flush(slot ^ 1);
        } catch (...) {
            cudaStreamSynchronize(C.stream);
            cudaEventDestroy(done[0]);
            cudaEventDestroy(done[1]);
            throw;
        }
        cudaEventDestroy(done[0]);
        cudaEventDestroy(done[1]);
    }
    if (fclose(F.f) != 0) {
        F.f = nullptr;
        throw Error(SSP_ERR_IO, "write failed");
    }
    F.f = nullptr;
}

// ---------------------------------------------------------------- edge lists
// edge_list_to_matrix_market (utils.rs:413-526) on the device: the body's lines are indexed and parsed in
// parallel, the (min, max) pairs sorted stably (so the first weight of a repeated pair wins), and the lines
// "i j w" formatted with w as Rust displays an f64.  Anything the per-line parser does not mirror exactly
// (signs, endpoints of 2^32 or more, separators other than spaces and tabs, a malformed line, a weight whose
// shortest text needs the host) sends the whole file to the host converter, which then writes the same bytes
// or reports the same error.  Weights the exact converter cannot read (more than 19 digits, inf, hex, trailing
// text) are read by strtod on the host from the line's own bytes, as the host converter reads them.
namespace {
enum : int32_t { EL_BLANK = 0, EL_ENTRY = 1, EL_HOST = 2 };
constexpr int EL_WSLOT = 48;  // bytes per formatted weight

__device__ __forceinline__ bool el_digit(char c) { return c >= '0' && c <= '9'; }

// kind[l]; for entries key = min << 32 | max, the weight (or wfix[l] = 1 and wpos[l] = its first byte)
__global__ void k_parse_edge_lines(const char* __restrict__ buf, int64_t size, const int64_t* __restrict__ starts,
                                   int64_t nlines, double defw, int32_t* __restrict__ kind,
                                   uint64_t* __restrict__ key, double* __restrict__ wt, int32_t* __restrict__ wfix,
                                   int64_t* __restrict__ wpos) {
    const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlines) return;
    const char* p = buf + starts[l];
    const char* e = buf + (l + 1 < nlines ? starts[l + 1] - 1 : size);  // excludes the newline
    wfix[l] = 0;
    // blank: nothing but spaces, tabs and carriage returns (the host converter's test)
    const char* q = p;
    while (q < e && (*q == ' ' || *q == '\t' || *q == '\r')) q++;
    if (q >= e) {
        kind[l] = EL_BLANK;
        return;
    }
    kind[l] = EL_HOST;
    uint64_t ep[2];
    for (int k = 0; k < 2; k++) {
        if (k == 1) {
            if (q >= e || (*q != ' ' && *q != '\t')) return;
            while (q < e && (*q == ' ' || *q == '\t')) q++;
        }
        if (q >= e || !el_digit(*q)) return;
        uint64_t v = 0;
        int nd = 0;
        for (; q < e && el_digit(*q); q++, nd++) {
            if (nd == 19) return;  // might not fit: the host reads it
            v = v * 10 + (uint64_t)(*q - '0');
        }
        ep[k] = v;
    }
    const uint64_t i = ep[0] < ep[1] ? ep[0] : ep[1], j = ep[0] < ep[1] ? ep[1] : ep[0];
    if (j >> 32) return;
    double w = defw;
    if (q < e && *q != '\r') {
        if (*q != ' ' && *q != '\t') return;  // text glued to the second endpoint
        while (q < e && (*q == ' ' || *q == '\t')) q++;
        if (q < e && *q != '\r') {
            const char* t = q;
            while (q < e && !is_space(*q)) q++;
            if (q == t) return;  // a vertical tab or form feed: the host converter's strtod rules
            if (dec::parse_decimal(t, q, &w) != dec::PARSE_OK) {
                wfix[l] = 1;
                wpos[l] = t - buf;
                w = 0.0;
            }
        }
    }
    key[l] = i << 32 | j;
    wt[l] = w;
    kind[l] = EL_ENTRY;
}

__global__ void k_el_flags(int64_t nlines, const int32_t* __restrict__ kind, int32_t* __restrict__ isent,
                           int32_t* __restrict__ nhost) {
    const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlines) return;
    isent[l] = kind[l] == EL_ENTRY;
    if (kind[l] == EL_HOST) atomicAdd(nhost, 1);
}

// entries in line order (their sort payload: the entry index), and the lines whose weight strtod reads
__global__ void k_el_gather(int64_t nlines, const int32_t* __restrict__ kind, const int64_t* __restrict__ rank,
                            const uint64_t* __restrict__ lkey, const double* __restrict__ lw,
                            const int32_t* __restrict__ wfix, int64_t nent, uint64_t* __restrict__ ekey,
                            int32_t* __restrict__ eidx, double* __restrict__ ew, int32_t* __restrict__ nfix,
                            int64_t* __restrict__ fixline, int32_t fixcap, unsigned long long* __restrict__ err) {
    const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlines || kind[l] != EL_ENTRY) return;
    const int64_t r = rank[l];
    if (r < 0 || r >= nent) {
        check_fail(err, 7, l);
        return;
    }
    ekey[r] = lkey[l];
    eidx[r] = (int32_t)r;
    ew[r] = lw[l];
    if (wfix[l]) {
        const int32_t t = atomicAdd(nfix, 1);
        if (t < fixcap) fixline[t] = l;
    }
}

// after the sort: the first entry of each pair, its weight formatted, its line's length
__global__ void k_el_format(int64_t nent, const uint64_t* __restrict__ skey, const int32_t* __restrict__ sidx,
                            const double* __restrict__ ew, int32_t* __restrict__ head, char* __restrict__ wtxt,
                            int32_t* __restrict__ llen, int32_t* __restrict__ nmiss) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nent) return;
    const bool h = t == 0 || skey[t] != skey[t - 1];
    head[t] = h;
    llen[t] = 0;
    if (!h) return;
    char* o = wtxt + t * EL_WSLOT;
    const int len = dec::format_shortest_fixed(ew[sidx[t]], o, EL_WSLOT);
    if (len < 0) {
        atomicAdd(nmiss, 1);
        return;
    }
    const uint64_t k = skey[t];
    llen[t] = dec_len((int64_t)(k >> 32)) + 1 + dec_len((int64_t)(k & 0xffffffffu)) + 1 + len + 1;
}

__global__ void k_el_write(int64_t nent, const uint64_t* __restrict__ skey, const int32_t* __restrict__ head,
                           const char* __restrict__ wtxt, const int32_t* __restrict__ llen,
                           const int64_t* __restrict__ loff, char* __restrict__ out, int64_t out_bytes,
                           unsigned long long* __restrict__ err) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nent || !head[t]) return;
    const uint64_t k = skey[t];
    const int64_t at = loff[t];
    if (at < 0 || at + llen[t] > out_bytes) {
        check_fail(err, 8, t);
        return;
    }
    char* o = out + at;
    o = put_int(o, (int64_t)(k >> 32));
    *o++ = ' ';
    o = put_int(o, (int64_t)(k & 0xffffffffu));
    *o++ = ' ';
    const int wl = llen[t] - (int)(o - (out + at)) - 1;
    for (int i = 0; i < wl; i++) o[i] = wtxt[t * EL_WSLOT + i];
    o[wl] = '\n';
}
}  // namespace

// false: the host converter must run (it then writes the same file or reports the same error)
bool edgelist_to_mtx_device(Context& C, const char* in_path, const char* out_path, double default_weight) {
    File F;
    F.f = fopen(in_path, "rb");
    if (!F.f) return false;
    // the first line "<num_nodes> <num_edges>", read as the host converter reads it
    std::string first;
    {
        char b[4096];
        for (;;) {
            if (!fgets(b, sizeof b, F.f)) break;
            first += b;
            if (!first.empty() && first.back() == '\n') break;
        }
    }
    unsigned long long n_nodes = 0, n_decl = 0;
    if (first.empty() || sscanf(first.c_str(), "%llu %llu", &n_nodes, &n_decl) != 2) return false;
    const long body = ftell(F.f);
    struct stat st;
    if (body < 0 || fstat(fileno(F.f), &st) != 0) return false;
    const int64_t size = (int64_t)st.st_size - body;
    Workspace& W = C.ws;
    const std::string tag = "edl";
    auto nm = [&](const char* s) { return tag + "_" + s; };
    unsigned long long* derr = W.get_t<unsigned long long>(nm("err"), 1);
    SSP_CUDA(cudaMemsetAsync(derr, 0xff, sizeof(unsigned long long), C.stream));
    char* dbuf = W.get_t<char>(nm("text"), (size_t)std::max<int64_t>(size, 1));
    upload_body(C, F.f, size, dbuf, in_path);
    int64_t* starts = nullptr;
    const int64_t nlines = line_index(C, dbuf, size, tag, derr, &starts);
    int32_t* kind = W.get_t<int32_t>(nm("kind"), nlines);
    uint64_t* lkey = W.get_t<uint64_t>(nm("lkey"), nlines);
    double* lw = W.get_t<double>(nm("lw"), nlines);
    int32_t* wfix = W.get_t<int32_t>(nm("wfix"), nlines);
    int64_t* wpos = W.get_t<int64_t>(nm("wpos"), nlines);
    const unsigned lb = (unsigned)ceil_div<int64_t>(nlines, 256);
    k_parse_edge_lines<<<lb, 256, 0, C.stream>>>(dbuf, size, starts, nlines, default_weight, kind, lkey, lw, wfix,
                                                 wpos);
    SSP_CHECK_LAUNCH();
    int32_t* isent = W.get_t<int32_t>(nm("isent"), nlines);
    int64_t* rank = W.get_t<int64_t>(nm("rank"), nlines + 1);
    int32_t* cnts = W.get_t<int32_t>(nm("cnts"), 4);  // host lines, weights for strtod, weights to format
    SSP_CUDA(cudaMemsetAsync(cnts, 0, sizeof(int32_t) * 4, C.stream));
    k_el_flags<<<lb, 256, 0, C.stream>>>(nlines, kind, isent, cnts);
    SSP_CHECK_LAUNCH();
    exclusive_scan_i32_to_i64(C, isent, rank, nlines, rank + nlines);
    C.kernels_launched += 2;
    const int64_t nent = read_i64(C, rank + nlines);
    int32_t hc[4];
    SSP_CUDA(cudaMemcpyAsync(hc, cnts, sizeof hc, cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    if (hc[0] != 0 || nent >= (int64_t)INT32_MAX) return false;
    const int64_t ne = std::max<int64_t>(nent, 1);
    uint64_t* ekey = W.get_t<uint64_t>(nm("ekey"), ne);
    int32_t* eidx = W.get_t<int32_t>(nm("eidx"), ne);
    double* ew = W.get_t<double>(nm("ew"), ne);
    int64_t* fixline = W.get_t<int64_t>(nm("fix"), HOST_FIX_CAP);
    k_el_gather<<<lb, 256, 0, C.stream>>>(nlines, kind, rank, lkey, lw, wfix, nent, ekey, eidx, ew, cnts + 1, fixline,
                                          HOST_FIX_CAP, derr);
    SSP_CHECK_LAUNCH();
    C.kernels_launched++;
    stage_check(C, derr, "edge gather");
    SSP_CUDA(cudaMemcpyAsync(hc, cnts, sizeof hc, cudaMemcpyDeviceToHost, C.stream));
    SSP_CUDA(cudaStreamSynchronize(C.stream));
    const int32_t nfix = hc[1];
    if (nfix > HOST_FIX_CAP) return false;
    if (nfix > 0) {
        // strtod on the host, from each line's weight to the line's end (the host converter's reading)
        std::vector<int64_t> lines(nfix);
        SSP_CUDA(cudaMemcpyAsync(lines.data(), fixline, sizeof(int64_t) * nfix, cudaMemcpyDeviceToHost, C.stream));
        SSP_CUDA(cudaStreamSynchronize(C.stream));
        for (int64_t l : lines) {
            int64_t hp[3] = {0, 0, 0};
            SSP_CUDA(cudaMemcpyAsync(&hp[0], wpos + l, sizeof(int64_t), cudaMemcpyDeviceToHost, C.stream));
            if (l + 1 < nlines)
                SSP_CUDA(cudaMemcpyAsync(&hp[1], starts + l + 1, sizeof(int64_t), cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaMemcpyAsync(&hp[2], rank + l, sizeof(int64_t), cudaMemcpyDeviceToHost, C.stream));
            SSP_CUDA(cudaStreamSynchronize(C.stream));
            const int64_t end = l + 1 < nlines ? hp[1] - 1 : size;
            std::string text((size_t)std::max<int64_t>(end - hp[0], 0), '\0');
            if (!text.empty()) {
                SSP_CUDA(cudaMemcpyAsync(&text[0], dbuf + hp[0], text.size(), cudaMemcpyDeviceToHost, C.stream));
                SSP_CUDA(cudaStreamSynchronize(C.stream));
            }
            char* stop = nullptr;
            const double x = strtod(text.c_str(), &stop);
            if (stop == text.c_str()) return false;  // "bad weight": the host converter reports it
            SSP_CUDA(cudaMemcpyAsync(ew + hp[2], &x, sizeof(double), cudaMemcpyHostToDevice, C.stream));
        }
        SSP_CUDA(cudaStreamSynchronize(C.stream));
    }
    // stable sort by (min, max): the first occurrence of a pair leads its run
    int64_t U = 0;
    std::string body_text;
    if (nent > 0) {
        uint64_t* tk = W.get_t<uint64_t>(nm("tkey"), ne);
        int32_t* ti = W.get_t<int32_t>(nm("tidx"), ne);
        radix_sort_u64(C, ekey, eidx, nent, 64, tk, ti, derr);
        stage_check(C, derr, "edge sort");
        int32_t* head = W.get_t<int32_t>(nm("head"), ne);
        char* wtxt = W.get_t<char>(nm("wtxt"), (size_t)ne * EL_WSLOT);
        int32_t* llen = W.get_t<int32_t>(nm("llen"), ne);
        int64_t* loff = W.get_t<int64_t>(nm("loff"), ne + 1);
        const unsigned eb = (unsigned)ceil_div<int64_t>(nent, 256);
        k_el_format<<<eb, 256, 0, C.stream>>>(nent, ekey, eidx, ew, head, wtxt, llen, cnts + 2);
        SSP_CHECK_LAUNCH();
        exclusive_scan_i32_to_i64(C, llen, loff, nent, loff + nent);
        C.kernels_launched++;
        SSP_CUDA(cudaMemcpyAsync(hc, cnts, sizeof hc, cudaMemcpyDeviceToHost, C.stream));
        const int64_t bytes = read_i64(C, loff + nent);
        if (hc[2] != 0) return false;  // a weight whose text the device does not produce
        int64_t* hoff = W.get_t<int64_t>(nm("hoff"), ne + 1);
        exclusive_scan_i32_to_i64(C, head, hoff, nent, hoff + nent);
        U = read_i64(C, hoff + nent);
        char* dout = W.get_t<char>(nm("out"), (size_t)std::max<int64_t>(bytes, 1));
        k_el_write<<<eb, 256, 0, C.stream>>>(nent, ekey, head, wtxt, llen, loff, dout, bytes, derr);
        SSP_CHECK_LAUNCH();
        C.kernels_launched++;
        stage_check(C, derr, "edge write");
        body_text.resize((size_t)bytes);
        if (bytes) copy_d2h(C, &body_text[0], dout, (size_t)bytes);
        SSP_CUDA(cudaStreamSynchronize(C.stream));
    }
    FILE* o = fopen(out_path, "w");
    if (!o) return false;
    fprintf(o, "%%%%MatrixMarket matrix coordinate real symmetric\n%% Converted from %s\n%llu %llu %lld\n", in_path,
            n_nodes, n_nodes, (long long)U);
    const bool ok = fwrite(body_text.data(), 1, body_text.size(), o) == body_text.size();
    if (fclose(o) != 0 || !ok) throw Error(SSP_ERR_IO, std::string("error writing ") + out_path);
    return true;
}

}  // namespace ssp
