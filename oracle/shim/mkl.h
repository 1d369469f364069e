/* mkl.h stand-in - TEST INFRASTRUCTURE ONLY.  MKL is not installed here, so
 * the reference's MKL CSR rows (intSpmv_main.c:461-569) cannot run; these
 * declarations only let the reference translation unit compile, and abort if
 * one is ever called.  No MKL arithmetic is reproduced. */
#ifndef REF_SHIM_MKL_H
#define REF_SHIM_MKL_H
#include <stdio.h>
#include <stdlib.h>
typedef int MKL_INT;
static inline void ref_shim_no_mkl(const char *f) {
  fprintf(stderr, "MKL is not available in this build (%s)\n", f);
  abort();
}
static inline void mkl_cspblas_dcsrgemv(const char *t, const unsigned int *m, const double *a,
                                        const unsigned int *ia, const unsigned int *ja,
                                        const double *x, double *y) {
  (void)t; (void)m; (void)a; (void)ia; (void)ja; (void)x; (void)y;
  ref_shim_no_mkl("mkl_cspblas_dcsrgemv");
}
#endif
