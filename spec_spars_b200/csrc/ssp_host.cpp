// ssp_host.cpp -- host-side I/O and synthetic graphs.
//
// read_mtx / write_mtx restate utils::read_mtx / write_mtx (utils.rs:149-154,189-191): Matrix
// Market coordinate files, symmetric storage expanded, duplicates summed, CSC with sorted rows.
// Pattern files (which the reference cannot read, utils.rs:172-186) load with weight 1.
//
// Generators produce the symmetric adjacency of the synthetic graphs used by the benchmark
// configurations, seeded through Philox so every host builds the same graph.
#include <algorithm>
#include <cerrno>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "ssp_host.h"

namespace ssp {

static inline uint64_t mulhi(uint64_t a, uint64_t b) { return (uint64_t)(((unsigned __int128)a * b) >> 64); }
static void philox_host(uint64_t c0, uint64_t c1, uint64_t c2, uint64_t c3, uint64_t k0, uint64_t k1,
                        uint64_t out[4]) {
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += 0x9E3779B97F4A7C15ULL;
            k1 += 0xBB67AE8584CAA73BULL;
        }
        const uint64_t M0 = 0xD2E7470EE14C6C93ULL, M1 = 0xCA5A826395121157ULL;
        uint64_t lo0 = M0 * c0, hi0 = mulhi(M0, c0), lo1 = M1 * c2, hi1 = mulhi(M1, c2);
        uint64_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
static constexpr uint64_t STREAM_GEN = 0x47454e31ULL;
static inline double gen_u53(uint64_t seed, uint64_t a, uint64_t b) {
    uint64_t o[4];
    philox_host(a, b, 0, 0, seed, STREAM_GEN, o);
    return (double)(o[0] >> 11) * 0x1.0p-53;
}

void HostCsc::from_upper_edges(int64_t n_, const std::vector<int32_t>& a, const std::vector<int32_t>& b,
                               const std::vector<double>& w) {
    // edges (a < b) sorted by (b, a): CSC-upper order.  Emit both triangles.
    n = n_;
    const int64_t m = (int64_t)a.size();
    std::vector<int64_t> cnt(n + 1, 0);
    for (int64_t e = 0; e < m; e++) {
        cnt[a[e] + 1]++;
        cnt[b[e] + 1]++;
    }
    colptr.assign(n + 1, 0);
    for (int64_t v = 0; v < n; v++) colptr[v + 1] = colptr[v] + cnt[v + 1];
    rowidx.assign(colptr[n], 0);
    val.assign(colptr[n], 0.0);
    std::vector<int64_t> cur(colptr.begin(), colptr.end() - 1);
    // column c: rows < c are edges (r, c) with b == c in order of r; rows > c are edges (c, v) in order of v.
    // Edges sorted by (b, a) visit every column's lower-row entries before any later column, and a
    // vertex's upper entries (c, v) arrive in increasing v.
    for (int64_t e = 0; e < m; e++) {
        int32_t r = a[e], c = b[e];
        rowidx[cur[c]] = r;
        val[cur[c]++] = w[e];
        rowidx[cur[r]] = c;
        val[cur[r]++] = w[e];
    }
}

// ---------------------------------------------------------------- generators
void gen_grid2d(int64_t nx, int64_t ny, double w, HostCsc& out) {
    const int64_t n = nx * ny;
    std::vector<int32_t> a, b;
    std::vector<double> ww;
    // CSC-upper order: for each column c (ascending), rows r < c ascending: r = c - nx, c - 1
    for (int64_t c = 0; c < n; c++) {
        int64_t x = c % nx, y = c / nx;
        if (y > 0) { a.push_back((int32_t)(c - nx)); b.push_back((int32_t)c); ww.push_back(w); }
        if (x > 0) { a.push_back((int32_t)(c - 1)); b.push_back((int32_t)c); ww.push_back(w); }
    }
    out.from_upper_edges(n, a, b, ww);
}

// 7-point grid, weight 10^U(lo,hi) per edge, drawn from Philox(seed, smaller endpoint, direction)
void gen_grid3d(int64_t nx, int64_t ny, int64_t nz, double lo, double hi, uint64_t seed, HostCsc& out) {
    const int64_t n = nx * ny * nz, nxy = nx * ny;
    std::vector<int32_t> a, b;
    std::vector<double> ww;
    a.reserve(3 * n); b.reserve(3 * n); ww.reserve(3 * n);
    for (int64_t c = 0; c < n; c++) {
        int64_t x = c % nx, y = (c / nx) % ny, z = c / nxy;
        int64_t rows[3];
        int dirs[3];
        int cnt = 0;
        if (z > 0) { rows[cnt] = c - nxy; dirs[cnt++] = 2; }
        if (y > 0) { rows[cnt] = c - nx; dirs[cnt++] = 1; }
        if (x > 0) { rows[cnt] = c - 1; dirs[cnt++] = 0; }
        for (int i = 0; i < cnt; i++) {
            double u = gen_u53(seed, (uint64_t)rows[i], (uint64_t)dirs[i]);
            double wv = std::pow(10.0, lo + (hi - lo) * u);
            a.push_back((int32_t)rows[i]);
            b.push_back((int32_t)c);
            ww.push_back(wv);
        }
    }
    out.from_upper_edges(n, a, b, ww);
}

// Erdos-Renyi G(n, p), p = avg_degree/(n-1), by geometric skipping over the pairs (w < v) in
// order of v then w (Batagelj & Brandes 2005); weights U[wlo, whi] rounded to float.
void gen_er(int64_t n, double avg_degree, double wlo, double whi, uint64_t seed, HostCsc& out) {
    const double p = std::min(1.0, avg_degree / (double)(n - 1));
    std::vector<int32_t> a, b;
    std::vector<double> ww;
    const int64_t expect = (int64_t)(p * (double)n * (double)(n - 1) / 2.0 * 1.05) + 16;
    a.reserve(expect); b.reserve(expect); ww.reserve(expect);
    const double lp = std::log1p(-p);
    int64_t v = 1, w = -1;
    uint64_t draw = 0;
    while (v < n) {
        double u = gen_u53(seed, draw++, 0);
        int64_t skip = (p >= 1.0) ? 0 : (int64_t)std::floor(std::log1p(-u) / lp);
        w += 1 + skip;
        while (w >= v && v < n) {
            w -= v;
            v++;
        }
        if (v < n) {
            double uw = gen_u53(seed, draw++, 1);
            float wf = (float)(wlo + (whi - wlo) * uw);
            a.push_back((int32_t)w);
            b.push_back((int32_t)v);
            ww.push_back((double)wf);
        }
    }
    out.from_upper_edges(n, a, b, ww);
}

// Random geometric graph: n points uniform in the unit square (Philox counters (i, 2) and (i, 3)), an edge
// between every pair closer than r = sqrt(avg_degree / (pi n)); weight uniform [wlo, whi] rounded to FP32
// from the counter (a * n + b, 4).  Pairs are found through a grid of r-sized cells.
void gen_rgg(int64_t n, double avg_degree, double wlo, double whi, uint64_t seed, HostCsc& out) {
    const double r = std::sqrt(avg_degree / (M_PI * (double)n));
    std::vector<double> px(n), py(n);
    for (int64_t i = 0; i < n; i++) {
        px[i] = gen_u53(seed, (uint64_t)i, 2);
        py[i] = gen_u53(seed, (uint64_t)i, 3);
    }
    const int64_t g = std::max<int64_t>(1, std::min<int64_t>((int64_t)(1.0 / r), 1 << 15));
    auto cell = [&](double x) { return std::min<int64_t>(g - 1, (int64_t)(x * (double)g)); };
    std::vector<int64_t> start(g * g + 1, 0), order(n);
    for (int64_t i = 0; i < n; i++) start[cell(py[i]) * g + cell(px[i]) + 1]++;
    for (int64_t c = 0; c < g * g; c++) start[c + 1] += start[c];
    std::vector<int64_t> fill(start.begin(), start.end() - 1);
    for (int64_t i = 0; i < n; i++) order[fill[cell(py[i]) * g + cell(px[i])]++] = i;
    std::vector<std::pair<int32_t, int32_t>> e;  // (b, a), a < b
    const double r2 = r * r;
    for (int64_t i = 0; i < n; i++) {
        const int64_t cx = cell(px[i]), cy = cell(py[i]);
        for (int64_t yy = std::max<int64_t>(0, cy - 1); yy <= std::min<int64_t>(g - 1, cy + 1); yy++)
            for (int64_t xx = std::max<int64_t>(0, cx - 1); xx <= std::min<int64_t>(g - 1, cx + 1); xx++)
                for (int64_t t = start[yy * g + xx]; t < start[yy * g + xx + 1]; t++) {
                    const int64_t j = order[t];
                    if (j <= i) continue;
                    const double dx = px[i] - px[j], dy = py[i] - py[j];
                    if (dx * dx + dy * dy < r2) e.push_back({(int32_t)j, (int32_t)i});
                }
    }
    std::sort(e.begin(), e.end());
    std::vector<int32_t> a(e.size()), b(e.size());
    std::vector<double> w(e.size());
    for (size_t t = 0; t < e.size(); t++) {
        b[t] = e[t].first;
        a[t] = e[t].second;
        const double u = gen_u53(seed, (uint64_t)a[t] * (uint64_t)n + (uint64_t)b[t], 4);
        w[t] = (double)(float)(wlo + (whi - wlo) * u);
    }
    out.from_upper_edges(n, a, b, w);
}

// R-MAT graph: edge_factor * 2^scale directed samples; each picks its quadrant bit by bit with probabilities
// (a, b, c, 1 - a - b - c) from Philox counters (sample, bit) in stream 5.  Self-loops are dropped, pairs are
// made undirected and deduplicated, each kept pair gets a LogNormal(0, 1) weight (Box-Muller from the
// counter (min * 2^scale + max, 6), rounded to FP32), and only the largest connected component is kept, its
// vertices renumbered in increasing order.
// Runs fn(t, lo, hi) over [0, count) split into contiguous ranges, one per host thread.
template <class Fn>
static void parallel_ranges(uint64_t count, Fn fn) {
    const unsigned hw = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    const uint64_t T = std::max<uint64_t>(1, std::min<uint64_t>(hw, count / 65536 + 1));
    std::vector<std::thread> th;
    for (uint64_t t = 0; t < T; t++)
        th.emplace_back([&, t] { fn(t, count * t / T, count * (t + 1) / T); });
    for (auto& x : th) x.join();
}

// Sorts in parallel: contiguous chunks sorted on their own threads, then merged pairwise (the result is
// the sorted sequence, whatever the thread count).
static void parallel_sort(std::vector<uint64_t>& v) {
    const unsigned hw = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    size_t parts = 1;
    while (parts * 2 <= hw && v.size() / (parts * 2) >= (1u << 20)) parts *= 2;
    std::vector<size_t> cut(parts + 1);
    for (size_t i = 0; i <= parts; i++) cut[i] = v.size() * i / parts;
    {
        std::vector<std::thread> th;
        for (size_t i = 0; i < parts; i++) th.emplace_back([&, i] { std::sort(v.begin() + cut[i], v.begin() + cut[i + 1]); });
        for (auto& x : th) x.join();
    }
    std::vector<uint64_t> tmp(v.size());
    for (size_t w = 1; w < parts; w *= 2) {
        std::vector<std::thread> th;
        for (size_t i = 0; i + w < parts; i += 2 * w) {
            const size_t lo = cut[i], mid = cut[i + w], hi = cut[std::min(parts, i + 2 * w)];
            th.emplace_back([&, lo, mid, hi] { std::merge(v.begin() + lo, v.begin() + mid, v.begin() + mid, v.begin() + hi,
                                                          tmp.begin() + lo); });
        }
        for (auto& x : th) x.join();
        // ranges left without a partner keep their place
        for (size_t i = 0; i < parts; i += 2 * w)
            if (i + w >= parts) std::copy(v.begin() + cut[i], v.begin() + cut[parts], tmp.begin() + cut[i]);
        v.swap(tmp);
    }
}

// R-MAT (Chakrabarti, Zhan, Faloutsos 2004): each of edge_factor * 2^scale samples picks a quadrant per bit
// level with probabilities (a, b, c, 1 - a - b - c), from Philox(seed, sample * 64 + level).  Self-loops are
// dropped, pairs symmetrized and deduplicated, the largest connected component kept (vertices renumbered in
// order), weights LogNormal(0, 1) rounded to FP32 from Philox counters of the pair.  Samples and weights are
// drawn on all host threads; every value depends only on its own counter, so the graph does not depend on
// the thread count.
void gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed, HostCsc& out) {
    const uint64_t nv = 1ull << scale;
    const uint64_t samples = (uint64_t)edge_factor << scale;
    const uint64_t NONE = ~0ull;
    std::vector<uint64_t> keys(samples);
    parallel_ranges(samples, [&](uint64_t, uint64_t lo, uint64_t hi) {
        for (uint64_t t = lo; t < hi; t++) {
            uint64_t u = 0, v = 0;
            for (int32_t bit = 0; bit < scale; bit++) {
                const double r = gen_u53(seed, t * 64 + (uint64_t)bit, 5);
                const int q = r < a ? 0 : r < a + b ? 1 : r < a + b + c ? 2 : 3;
                u = (u << 1) | (uint64_t)(q >> 1);
                v = (v << 1) | (uint64_t)(q & 1);
            }
            keys[t] = u == v ? NONE : std::min(u, v) * nv + std::max(u, v);
        }
    });
    parallel_sort(keys);
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    if (!keys.empty() && keys.back() == NONE) keys.pop_back();
    // largest connected component by union-find (smaller root wins, so labels are deterministic)
    std::vector<uint64_t> parent(nv);
    for (uint64_t i = 0; i < nv; i++) parent[i] = i;
    auto find = [&](uint64_t x) {
        while (parent[x] != x) x = parent[x] = parent[parent[x]];
        return x;
    };
    for (uint64_t k : keys) {
        uint64_t ra = find(k / nv), rb = find(k % nv);
        if (ra != rb) parent[std::max(ra, rb)] = std::min(ra, rb);
    }
    std::vector<uint64_t> size(nv, 0);
    for (uint64_t i = 0; i < nv; i++) size[find(i)]++;
    uint64_t best = 0;
    for (uint64_t i = 0; i < nv; i++)
        if (size[i] > size[best]) best = i;
    std::vector<int64_t> newid(nv, -1);
    int64_t n = 0;
    for (uint64_t i = 0; i < nv; i++)
        if (find(i) == best) newid[i] = n++;
    // kept pairs in CSC-upper order (by (hi, lo)) with their weights
    std::vector<std::pair<int64_t, int64_t>> e;
    std::vector<uint64_t> ek;
    for (uint64_t k : keys) {
        const uint64_t lo = k / nv, hi = k % nv;
        if (newid[lo] < 0) continue;
        e.push_back({newid[hi], newid[lo]});
        ek.push_back(k);
    }
    std::vector<size_t> order(e.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](size_t x, size_t y) { return e[x] < e[y]; });
    std::vector<int32_t> va(e.size()), vb(e.size());
    std::vector<double> w(e.size());
    parallel_ranges(order.size(), [&](uint64_t, uint64_t lo, uint64_t hi) {
        for (uint64_t t = lo; t < hi; t++) {
            const size_t i = order[t];
            vb[t] = (int32_t)e[i].first;
            va[t] = (int32_t)e[i].second;
            const double u1 = gen_u53(seed, ek[i], 6), u2 = gen_u53(seed ^ 0x9e3779b97f4a7c15ull, ek[i], 6);
            const double z = std::sqrt(-2.0 * std::log(1.0 - u1)) * std::cos(2.0 * M_PI * u2);
            w[t] = (double)(float)std::exp(z);
        }
    });
    out.from_upper_edges(n, va, vb, w);
}

// An f64 as Rust's Display writes it (the weights of edge_list_to_matrix_market, utils.rs:519): the shortest
// digits that read back as v (the closest such digits), placed without an exponent and padded with zeros
// (2^70 -> "1180591620717411300000", 5e-324 -> "0.000...005"); "NaN", "inf", "-inf"; -0.0 -> "-0".  The digits
// come from to_chars' shortest scientific form, which picks the same digits.
std::string rust_display_f64(double v) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v < 0 ? "-inf" : "inf";
    char sci[64];
    auto r = std::to_chars(sci, sci + sizeof sci - 1, v, std::chars_format::scientific);
    *r.ptr = 0;
    std::string out;
    const char* p = sci;
    if (*p == '-') {
        out += '-';
        p++;
    }
    std::string dig;
    for (; *p && *p != 'e'; p++)
        if (*p != '.') dig += *p;
    const int ex = *p == 'e' ? atoi(p + 1) : 0;  // value = d.ddd * 10^ex
    while (dig.size() > 1 && dig.back() == '0') dig.pop_back();
    if (dig == "0") return out + "0";
    const int L = (int)dig.size();
    const int ip = ex + 1;  // digits before the point
    if (ip >= L) {
        out += dig;
        out.append((size_t)(ip - L), '0');
    } else if (ip > 0) {
        out += dig.substr(0, (size_t)ip);
        out += '.';
        out += dig.substr((size_t)ip);
    } else {
        out += "0.";
        out.append((size_t)(-ip), '0');
        out += dig;
    }
    return out;
}

// Edge list -> Matrix Market (edge_list_to_matrix_market, utils.rs:413-526).  The first line holds
// "<num_nodes> <num_edges>" (the edge count is not used); each further non-blank line "u v [w]", w defaulting
// to default_weight.  Pairs are stored as (min, max); for repeated pairs the first weight wins.  The output is
// a symmetric real coordinate file with the pairs sorted, indices written as read, and weights in the
// shortest round-trip digits without an exponent (how Rust displays an f64, rust_display_f64).
int edgelist_to_mtx(const char* in_path, const char* out_path, double default_weight, std::string& err) {
    FILE* f = fopen(in_path, "r");
    if (!f) {
        err = std::string("cannot open ") + in_path;
        return -1;
    }
    std::vector<char> buf(1 << 16);
    std::string line;
    auto getline = [&](std::string& out) -> bool {
        out.clear();
        for (;;) {
            if (!fgets(buf.data(), (int)buf.size(), f)) return !out.empty();
            out += buf.data();
            if (!out.empty() && out.back() == '\n') return true;
        }
    };
    if (!getline(line)) {
        fclose(f);
        err = "empty input file";
        return -1;
    }
    unsigned long long n_nodes = 0, n_decl = 0;
    if (sscanf(line.c_str(), "%llu %llu", &n_nodes, &n_decl) != 2) {
        fclose(f);
        err = "first line must hold the node and edge counts";
        return -1;
    }
    std::vector<std::pair<std::pair<uint64_t, uint64_t>, double>> edges;
    std::vector<std::pair<std::pair<uint64_t, uint64_t>, size_t>> keys;
    size_t lineno = 1;
    while (getline(line)) {
        lineno++;
        size_t p = line.find_first_not_of(" \t\r\n");
        if (p == std::string::npos) continue;
        const char* c = line.c_str() + p;
        char* end = nullptr;
        errno = 0;
        const unsigned long long u = strtoull(c, &end, 10);
        if (end == c || errno) {
            fclose(f);
            err = "line " + std::to_string(lineno) + ": missing first endpoint";
            return -1;
        }
        c = end;
        const unsigned long long v = strtoull(c, &end, 10);
        if (end == c || errno) {
            fclose(f);
            err = "line " + std::to_string(lineno) + ": missing second endpoint";
            return -1;
        }
        c = end;
        while (*c == ' ' || *c == '\t') c++;
        double w = default_weight;
        if (*c && *c != '\n' && *c != '\r') {
            w = strtod(c, &end);
            if (end == c) {
                fclose(f);
                err = "line " + std::to_string(lineno) + ": bad weight";
                return -1;
            }
        }
        const uint64_t i = std::min(u, v), j = std::max(u, v);
        keys.push_back({{i, j}, edges.size()});
        edges.push_back({{i, j}, w});
    }
    fclose(f);
    // first occurrence wins: stable order by (pair, position), keep the first of each pair
    std::sort(keys.begin(), keys.end());
    FILE* o = fopen(out_path, "w");
    if (!o) {
        err = std::string("cannot write ") + out_path;
        return -1;
    }
    size_t unique = 0;
    for (size_t t = 0; t < keys.size(); t++)
        if (t == 0 || keys[t].first != keys[t - 1].first) unique++;
    fprintf(o, "%%%%MatrixMarket matrix coordinate real symmetric\n%% Converted from %s\n%llu %llu %zu\n", in_path,
            n_nodes, n_nodes, unique);
    for (size_t t = 0; t < keys.size(); t++) {
        if (t > 0 && keys[t].first == keys[t - 1].first) continue;
        const double w = edges[keys[t].second].second;
        fprintf(o, "%llu %llu %s\n", (unsigned long long)keys[t].first.first,
                (unsigned long long)keys[t].first.second, rust_display_f64(w).c_str());
    }
    const bool ok = fclose(o) == 0;
    if (!ok) err = std::string("error writing ") + out_path;
    return ok ? 0 : -1;
}

// ---------------------------------------------------------------- Matrix Market
static bool lower_eq(const std::string& a, const char* b) {
    if (a.size() != strlen(b)) return false;
    for (size_t i = 0; i < a.size(); i++)
        if (tolower(a[i]) != b[i]) return false;
    return true;
}

int read_mtx(const char* path, HostCsc& out, std::string& err) {
    FILE* f = fopen(path, "r");
    if (!f) {
        err = std::string("cannot open ") + path;
        return -1;
    }
    char line[4096];
    if (!fgets(line, sizeof line, f)) {
        fclose(f);
        err = "empty file";
        return -1;
    }
    char banner[64], object[64], format[64], field[64], sym[64];
    if (sscanf(line, "%63s %63s %63s %63s %63s", banner, object, format, field, sym) != 5 ||
        !lower_eq(banner, "%%matrixmarket") || !lower_eq(object, "matrix") || !lower_eq(format, "coordinate")) {
        fclose(f);
        err = "not a MatrixMarket coordinate matrix";
        return -1;
    }
    bool pattern = lower_eq(field, "pattern");
    if (!pattern && !lower_eq(field, "real") && !lower_eq(field, "integer") && !lower_eq(field, "double")) {
        fclose(f);
        err = std::string("unsupported field ") + field;
        return -1;
    }
    bool symmetric = lower_eq(sym, "symmetric");
    if (!symmetric && !lower_eq(sym, "general")) {
        fclose(f);
        err = std::string("unsupported symmetry ") + sym;
        return -1;
    }
    long long nr = 0, nc = 0, nnz = 0;
    while (fgets(line, sizeof line, f)) {
        if (line[0] == '%') continue;
        if (sscanf(line, "%lld %lld %lld", &nr, &nc, &nnz) == 3) break;
        fclose(f);
        err = "bad size line";
        return -1;
    }
    if (nr <= 0 || nr != nc || nnz < 0) {
        fclose(f);
        err = "matrix must be square";
        return -1;
    }
    std::vector<int64_t> I, J;
    std::vector<double> V;
    I.reserve(symmetric ? 2 * nnz : nnz);
    J.reserve(symmetric ? 2 * nnz : nnz);
    V.reserve(symmetric ? 2 * nnz : nnz);
    for (long long t = 0; t < nnz; t++) {
        long long i, j;
        double x = 1.0;
        int got;
        if (pattern) got = fscanf(f, "%lld %lld", &i, &j) == 2;
        else got = fscanf(f, "%lld %lld %lf", &i, &j, &x) == 3;
        if (!got || i < 1 || j < 1 || i > nr || j > nc) {
            fclose(f);
            err = "bad entry " + std::to_string(t);
            return -1;
        }
        I.push_back(i - 1);
        J.push_back(j - 1);
        V.push_back(x);
        if (symmetric && i != j) {
            I.push_back(j - 1);
            J.push_back(i - 1);
            V.push_back(x);
        }
    }
    fclose(f);
    // CSC: sort by (col, row), sum duplicates
    const int64_t n = nr;
    std::vector<int64_t> order(I.size());
    for (size_t t = 0; t < order.size(); t++) order[t] = (int64_t)t;
    std::sort(order.begin(), order.end(), [&](int64_t x, int64_t y) {
        return J[x] != J[y] ? J[x] < J[y] : (I[x] != I[y] ? I[x] < I[y] : x < y);
    });
    out.n = n;
    out.colptr.assign(n + 1, 0);
    out.rowidx.clear();
    out.val.clear();
    for (size_t t = 0; t < order.size(); t++) {
        int64_t o = order[t];
        if (!out.rowidx.empty() && t > 0 && J[order[t - 1]] == J[o] && I[order[t - 1]] == I[o]) {
            out.val.back() += V[o];
            continue;
        }
        out.rowidx.push_back((int32_t)I[o]);
        out.val.push_back(V[o]);
        out.colptr[J[o] + 1]++;
    }
    for (int64_t c = 0; c < n; c++) out.colptr[c + 1] += out.colptr[c];
    return 0;
}

int write_mtx(const char* path, int64_t n, const int64_t* colptr, const int32_t* rowidx, const double* val,
              std::string& err) {
    FILE* f = fopen(path, "w");
    if (!f) {
        err = std::string("cannot open ") + path + " for writing";
        return -1;
    }
    fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n");
    fprintf(f, "%lld %lld %lld\n", (long long)n, (long long)n, (long long)colptr[n]);
    for (int64_t c = 0; c < n; c++)
        for (int64_t p = colptr[c]; p < colptr[c + 1]; p++)
            fprintf(f, "%d %lld %.17g\n", rowidx[p] + 1, (long long)(c + 1), val[p]);
    if (fclose(f) != 0) {
        err = "write failed";
        return -1;
    }
    return 0;
}

}  // namespace ssp
