// Minimal stand-ins for the cxx bridge types used by the reference's C++ sources, so that the
// reference solver can be compiled without Rust.  Test infrastructure only.
#pragma once
#include <cstring>
#include <string>
#include <vector>
namespace rust {
inline namespace cxxbridge1 {
template <class T>
struct Vec : std::vector<T> {
    using std::vector<T>::vector;
};
struct Str {
    const char* p;
    size_t n;
    Str(const char* s = "") : p(s), n(std::strlen(s)) {}
    const char* data() const { return p; }
    size_t size() const { return n; }
};
}  // namespace cxxbridge1
}  // namespace rust
