// ssp_host.h -- host-side containers, I/O and generators.
#pragma once
#include <stdint.h>
#include <string>
#include <vector>

namespace ssp {

struct HostCsc {
    int64_t n = 0;
    std::vector<int64_t> colptr;
    std::vector<int32_t> rowidx;
    std::vector<double> val;
    // build the symmetric matrix of edges (a[e] < b[e]) given in CSC-upper order (sorted by (b, a))
    void from_upper_edges(int64_t n, const std::vector<int32_t>& a, const std::vector<int32_t>& b,
                          const std::vector<double>& w);
};

void gen_grid2d(int64_t nx, int64_t ny, double w, HostCsc& out);
void gen_grid3d(int64_t nx, int64_t ny, int64_t nz, double lo, double hi, uint64_t seed, HostCsc& out);
void gen_er(int64_t n, double avg_degree, double wlo, double whi, uint64_t seed, HostCsc& out);
void gen_rgg(int64_t n, double avg_degree, double wlo, double whi, uint64_t seed, HostCsc& out);
void gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed, HostCsc& out);

int read_mtx(const char* path, HostCsc& out, std::string& err);
int edgelist_to_mtx(const char* in_path, const char* out_path, double default_weight, std::string& err);
// an f64 as Rust's Display writes it (shortest round-trip digits, no exponent)
std::string rust_display_f64(double v);
int write_mtx(const char* path, int64_t n, const int64_t* colptr, const int32_t* rowidx, const double* val,
              std::string& err);

}  // namespace ssp
