// Stand-in for the cxx-generated header of the reference crate: the bridged struct of src/lib.rs:81-85.
#pragma once
#include "rust/cxx.h"
struct FlattenedVec {
    rust::Vec<double> vec;
    size_t num_cols;
    size_t num_rows;
};
