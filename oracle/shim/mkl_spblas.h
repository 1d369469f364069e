/* mkl_spblas.h stand-in - TEST INFRASTRUCTURE ONLY (see shim/mkl.h). */
#ifndef REF_SHIM_MKL_SPBLAS_H
#define REF_SHIM_MKL_SPBLAS_H
#include "mkl.h"
typedef enum { SPARSE_STATUS_SUCCESS = 0, SPARSE_STATUS_NOT_SUPPORTED = 6 } sparse_status_t;
typedef enum { SPARSE_MATRIX_TYPE_GENERAL = 20, SPARSE_MATRIX_TYPE_SYMMETRIC = 21 } sparse_matrix_type_t;
typedef enum { SPARSE_FILL_MODE_UPPER = 41 } sparse_fill_mode_t;
typedef enum { SPARSE_DIAG_NON_UNIT = 50 } sparse_diag_type_t;
typedef enum { SPARSE_INDEX_BASE_ZERO = 0 } sparse_index_base_t;
typedef enum { SPARSE_OPERATION_NON_TRANSPOSE = 10 } sparse_operation_t;
struct matrix_descr { sparse_matrix_type_t type; sparse_fill_mode_t mode; sparse_diag_type_t diag; };
typedef struct ref_shim_sparse_matrix *sparse_matrix_t;
static inline sparse_status_t mkl_sparse_d_create_csr(sparse_matrix_t *h, sparse_index_base_t b,
    unsigned int r, unsigned int c, unsigned int *rs, unsigned int *re, unsigned int *ci, double *v) {
  (void)h; (void)b; (void)r; (void)c; (void)rs; (void)re; (void)ci; (void)v;
  ref_shim_no_mkl("mkl_sparse_d_create_csr");
  return SPARSE_STATUS_NOT_SUPPORTED;
}
static inline sparse_status_t mkl_sparse_d_mv(sparse_operation_t op, double a, sparse_matrix_t h,
    struct matrix_descr d, const double *x, double b, double *y) {
  (void)op; (void)a; (void)h; (void)d; (void)x; (void)b; (void)y;
  ref_shim_no_mkl("mkl_sparse_d_mv");
  return SPARSE_STATUS_NOT_SUPPORTED;
}
static inline sparse_status_t mkl_sparse_set_mv_hint(sparse_matrix_t h, sparse_operation_t op,
    struct matrix_descr d, MKL_INT n) {
  (void)h; (void)op; (void)d; (void)n;
  ref_shim_no_mkl("mkl_sparse_set_mv_hint");
  return SPARSE_STATUS_NOT_SUPPORTED;
}
static inline sparse_status_t mkl_sparse_optimize(sparse_matrix_t h) {
  (void)h;
  ref_shim_no_mkl("mkl_sparse_optimize");
  return SPARSE_STATUS_NOT_SUPPORTED;
}
#endif
