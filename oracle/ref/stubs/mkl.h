// Declarations of the Intel MKL entry points the reference solver calls (custom_cg.hpp), taken from
// MKL's public API documentation; implemented by mkl_rci_shim.cc.  Enum values are this harness's own.
#pragma once
#include <cstddef>
typedef int MKL_INT;
typedef enum { SPARSE_STATUS_SUCCESS = 0, SPARSE_STATUS_INVALID_VALUE = 3 } sparse_status_t;
typedef enum { SPARSE_OPERATION_NON_TRANSPOSE = 10, SPARSE_OPERATION_TRANSPOSE = 11 } sparse_operation_t;
typedef enum {
    SPARSE_MATRIX_TYPE_GENERAL = 20,
    SPARSE_MATRIX_TYPE_SYMMETRIC = 21,
    SPARSE_MATRIX_TYPE_TRIANGULAR = 23
} sparse_matrix_type_t;
typedef enum { SPARSE_FILL_MODE_LOWER = 40, SPARSE_FILL_MODE_UPPER = 41, SPARSE_FILL_MODE_FULL = 42 } sparse_fill_mode_t;
typedef enum { SPARSE_DIAG_NON_UNIT = 50, SPARSE_DIAG_UNIT = 51 } sparse_diag_type_t;
typedef enum { SPARSE_INDEX_BASE_ZERO = 0, SPARSE_INDEX_BASE_ONE = 1 } sparse_index_base_t;
struct matrix_descr {
    sparse_matrix_type_t type;
    sparse_fill_mode_t mode;
    sparse_diag_type_t diag;
};
struct sparse_matrix;
typedef struct sparse_matrix* sparse_matrix_t;

void dcg_init(const MKL_INT* n, const double* x, const double* b, MKL_INT* rci_request, MKL_INT* ipar, double* dpar,
              double* tmp);
void dcg_check(const MKL_INT* n, const double* x, const double* b, MKL_INT* rci_request, MKL_INT* ipar, double* dpar,
               double* tmp);
void dcg(const MKL_INT* n, double* x, const double* b, MKL_INT* rci_request, MKL_INT* ipar, double* dpar, double* tmp);
sparse_status_t mkl_sparse_d_create_csr(sparse_matrix_t* A, sparse_index_base_t indexing, MKL_INT rows, MKL_INT cols,
                                        MKL_INT* rows_start, MKL_INT* rows_end, MKL_INT* col_indx, double* values);
sparse_status_t mkl_sparse_d_mv(sparse_operation_t op, double alpha, const sparse_matrix_t A, struct matrix_descr descr,
                                const double* x, double beta, double* y);
sparse_status_t mkl_sparse_d_trsv(sparse_operation_t op, double alpha, const sparse_matrix_t A,
                                  struct matrix_descr descr, const double* x, double* y);
sparse_status_t mkl_sparse_destroy(sparse_matrix_t A);
double cblas_dnrm2(const MKL_INT n, const double* x, const MKL_INT incx);
