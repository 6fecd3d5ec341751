// ref_solve.cc -- runs the reference's own Laplacian solver (src/example.cc factorization_driver: parallel
// randomized Cholesky + MKL-style PCG, include/custom_cg.hpp) on a Laplacian and a set of right-hand
// sides read from a binary file.  Test infrastructure only: built into oracle/_ref/ by oracle/ref/Makefile
// straight from the reference's sources (which are not part of this repository) and used to check the
// oracle and time the reference's CPU path.
//
// Input file (little endian): "SSPR", i32 n, i32 k, i32 threads, i32 verbose, i64 nnz,
//   i32 colptr[n+1], i32 rowidx[nnz], f64 values[nnz]   -- the Laplacian, CSC, all entries
//   f64 rhs[k][n]                                          -- one right-hand side after another
// Output file: i32 status (0 = every column converged, 1 = the driver returned false, 2 = it threw),
//   f64 seconds (processor set-up + factorization + solves), i32 s, f64 starts[s] (seconds from the start to
//   the beginning of each PCG solve, recorded by the MKL shim), f64 x[k][n], then the exception text if any.
#include "spec_spars/src/example.cc"

#include <chrono>
#include <cstdio>
#include <cstring>

extern "C" int ssp_shim_solve_starts(const double** t);

namespace {
template <class T>
bool rd(FILE* f, T* p, size_t count) {
    return std::fread(p, sizeof(T), count, f) == count;
}
}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: ref_solve <input> <output>\n");
        return 64;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 65;
    char magic[4];
    int32_t hdr[4];
    int64_t nnz = 0;
    if (!rd(f, magic, 4) || std::memcmp(magic, "SSPR", 4) != 0 || !rd(f, hdr, 4) || !rd(f, &nnz, 1)) return 66;
    const int32_t n = hdr[0], k = hdr[1], threads = hdr[2], verbose = hdr[3];
    std::vector<int> colptr(n + 1), rowidx(nnz);
    std::vector<double> vals(nnz);
    std::vector<std::vector<double>> rhs(k, std::vector<double>(n)), sol(k, std::vector<double>(n, 0.0));
    if (!rd(f, colptr.data(), n + 1) || !rd(f, rowidx.data(), nnz) || !rd(f, vals.data(), nnz)) return 66;
    for (int j = 0; j < k; ++j)
        if (!rd(f, rhs[j].data(), n)) return 66;
    std::fclose(f);

    int32_t status = 0;
    std::string err;
    char path[8] = "";
    const auto t0 = std::chrono::steady_clock::now();
    try {
        sparse_matrix_processor<int, double> processor("ref_solve_input", n, n, std::move(colptr), std::move(rowidx),
                                                       std::move(vals), verbose != 0);
        const bool ok = factorization_driver<int, double>(processor, threads, path, true, rhs, sol, verbose != 0);
        status = ok ? 0 : 1;
    } catch (const std::exception& e) {
        status = 2;
        err = e.what();
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 67;
    std::fwrite(&status, sizeof status, 1, o);
    std::fwrite(&secs, sizeof secs, 1, o);
    const double* st = nullptr;
    const int32_t ns = ssp_shim_solve_starts(&st);
    const double base = std::chrono::duration<double>(t0.time_since_epoch()).count();
    std::fwrite(&ns, sizeof ns, 1, o);
    for (int32_t i = 0; i < ns; ++i) {
        const double rel = st[i] - base;
        std::fwrite(&rel, sizeof rel, 1, o);
    }
    for (int j = 0; j < k; ++j) std::fwrite(sol[j].data(), sizeof(double), n, o);
    std::fwrite(err.data(), 1, err.size(), o);
    std::fclose(o);
    return 0;
}
