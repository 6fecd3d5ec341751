// Stand-in for the fast_matrix_market reader: the harness builds matrices from arrays only, so the
// file constructor of the reference's sparse_matrix_processor is never used.
#pragma once
// The real header pulls in much of the standard library, which the reference's headers rely on.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <iomanip>
#include <istream>
#include <map>
#include <numeric>
#include <sstream>
#include <string>
#include <thread>
#include <tuple>
#include <stdexcept>
#include <vector>
namespace fast_matrix_market {
template <class IT, class VT>
void read_matrix_market_triplet(std::istream&, IT&, IT&, std::vector<IT>&, std::vector<IT>&, std::vector<VT>&) {
    throw std::runtime_error("matrix market files are not read by this harness");
}
}  // namespace fast_matrix_market
