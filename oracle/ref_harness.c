/*
 * ref_harness.c - TEST INFRASTRUCTURE ONLY: exposes the reference's own
 * static functions (builders, kernels, error metric) from a shared library so
 * tests can pin the oracle against the reference itself and bench.py's
 * reference arm can time the reference's CPU kernels.
 *
 * The reference source is compiled where it lies: REF_SOURCE names it (the
 * Makefile in this directory passes its path), `main` is renamed, and
 * shim/ref_shim.h is force-included so GCC accepts the ICC-only code.  Nothing
 * of the reference is copied here; every `ref_*` function below only calls
 * reference functions, with the argument conventions of the reference's own
 * test_* wrappers (cited per function).  Line numbers are intSpmv_main.c's.
 */
#include <stdio.h>

int ref_shim_zero = 1;
int ref_shim_tracking = 0;
int ref_shim_ntrack = 0;
void *ref_shim_track[REF_SHIM_MAX_TRACK];

#define main ref_main
#include REF_SOURCE
#undef main

#define REF_API __attribute__((visibility("default")))

static void ref_release_tracked(void) {
  for (int i = 0; i < ref_shim_ntrack; i++) free(ref_shim_track[i]);
  ref_shim_ntrack = 0;
}

/* Struct sizes, so callers can check their mirrors of M:183,306,400,429,615,771,1114. */
REF_API size_t ref_sizeof(int which) {
  switch (which) {
    case 0: return sizeof(str_matCSR);
    case 1: return sizeof(str_formatData);
    case 2: return sizeof(str_err);
    case 3: return sizeof(str_res);
    case 4: return sizeof(str_matAXC);
    case 5: return sizeof(str_matK1);
    case 6: return sizeof(str_matAXT);
    default: return 0;
  }
}

REF_API int ref_num_ite(void) { return NUM_ITE; }

/* printMatrixStats (M:253): fills rl and the stats; writes <path minus ext>.sta */
REF_API void ref_stats(const char *path, str_matCSR *csr) { printMatrixStats(path, csr); }

REF_API void ref_init_vec(UIN len, FPT *vec) { initVec(len, vec); }

REF_API void ref_build_csr(str_matCSR *csr, str_formatData *fd) { *fd = getFormatDataCSR(csr); }

REF_API void ref_build_axc(UIN ompNT, const str_matCSR *csr, const FPT *vec, str_matAXC *out,
                           str_formatData *fd) {
  ref_shim_zero = 1;
  *fd = getFormatDataAXC(ompNT, *csr, vec, out);
}

REF_API void ref_build_k1(const str_matCSR *csr, const FPT *vec, str_matK1 *out, str_formatData *fd) {
  ref_shim_zero = 1;
  *fd = getFormatDataK1(CHUNK_SIZE, *csr, vec, out);
}

REF_API void ref_build_axt(UIN ompNT, UIN bs, UIN thw, UIN th, const char *mode,
                           const str_matCSR *csr, const FPT *vec, str_matAXT *out,
                           str_formatData *fd) {
  ref_shim_zero = 1;
  *fd = getFormatDataAXT(ompNT, bs, thw, th, mode, *csr, vec, out);
}

REF_API void ref_cf_csr(const str_matCSR *csr, const FPT *vec, FPT *res) { cf_CSR(*csr, vec, res); }

REF_API void ref_int_axc(UIN ompNT, const str_matAXC *m, FPT *y) {
  int_axc(ompNT, m->nrows, m->ax, m->brp, y);
}

/* test_int_k1, M:980-1022: int_k1 into res[chunkNum*8], then orderArrayK1. */
REF_API void ref_int_k1(UIN ompNT, const str_matK1 *m, const FPT *vec, FPT *res, FPT *y) {
  int_k1(ompNT, m->chunkNum, m->val, m->col, m->chp, m->nmc, vec, res);
  orderArrayK1(ompNT, m->nrows, m->permi, res, y);
}

/* test_int_k1p, M:1070-1110: the tail mask of the last chunk, M:1077-1086. */
static __mmask8 ref_k1p_mask(const str_matK1 *m) {
  const UIN posDif = (m->chunkNum * CHUNK_SIZE) - m->nrows;
  return (__mmask8)(0xFFu >> posDif);
}
REF_API unsigned ref_k1p_mask_of(const str_matK1 *m) { return ref_k1p_mask(m); }
REF_API void ref_int_k1p(UIN ompNT, const str_matK1 *m, const FPT *vec, FPT *y) {
  int_k1p(ompNT, ref_k1p_mask(m), m->chunkNum, m->val, m->col, m->chp, m->nmc, m->permi, vec, y);
}

REF_API void ref_int_axt_noc_h1(UIN ompNT, const str_matAXT *m, FPT *y) {
  int_axt_noc_h1(ompNT, m->tileN, m->ax, m->sec, y);
}

REF_API void ref_int_axt_noc(UIN ompNT, const str_matAXT *m, FPT *y) {
  int_axt_noc(ompNT, m->tileN, m->tileH, m->ax, m->sec, y);
}

/* test_int_axt_com_h1, M:1570-1609: bn = ceil(tileN*8 / bs).  The kernel's
 * per-call scratch (M:1529-1530) is freed after the call. */
REF_API void ref_int_axt_com_h1(UIN ompNT, UIN bs, const str_matAXT *m, FPT *y) {
  const UIN bn = ((m->tileN * HBRICK_SIZE) + bs - 1) / bs;
  ref_shim_zero = 0;
  ref_shim_tracking = 1;
  int_axt_com_h1(ompNT, bn, bs, m->log, m->tileHW, m->tileN, m->lenAX, m->lenSEC, m->ax, m->sec, y);
  ref_shim_tracking = 0;
  ref_shim_zero = 1;
  ref_release_tracked();
}

REF_API void ref_get_errors(UIN len, const FPT *ar, const FPT *ac, str_err *e) { getErrors(len, ar, ac, e); }

/*
 * Timing, as the reference's test_* wrappers time (gettimeofday around each
 * kernel call, mean over `iters`; y zeroed outside the timed region for the
 * accumulating AXT kernels, M:1421,1492,1591).  Returns seconds per call.
 * kind: 0 cf_CSR, 1 int_axc, 2 int_k1 (+orderArrayK1 time in *ot),
 * 3 int_k1p, 4 int_axt_noc_h1, 5 int_axt_noc, 6 int_axt_com_h1.
 */
REF_API double ref_time_kernel(int kind, UIN ompNT, const void *mat, UIN bs, const FPT *vec,
                               FPT *work, FPT *y, int iters, double *ot) {
  struct timeval t1, t2;
  double tt = 0.0, to = 0.0;
  for (int i = 0; i < iters; i++) {
    switch (kind) {
      case 0: {
        const str_matCSR *m = (const str_matCSR *)mat;
        GT(t1); cf_CSR(*m, vec, y); GT(t2);
        tt += measureTime(t2, t1);
      } break;
      case 1: {
        const str_matAXC *m = (const str_matAXC *)mat;
        GT(t1); int_axc(ompNT, m->nrows, m->ax, m->brp, y); GT(t2);
        tt += measureTime(t2, t1);
      } break;
      case 2: {
        const str_matK1 *m = (const str_matK1 *)mat;
        GT(t1); int_k1(ompNT, m->chunkNum, m->val, m->col, m->chp, m->nmc, vec, work); GT(t2);
        tt += measureTime(t2, t1);
        GT(t1); orderArrayK1(ompNT, m->nrows, m->permi, work, y); GT(t2);
        to += measureTime(t2, t1);
      } break;
      case 3: {
        const str_matK1 *m = (const str_matK1 *)mat;
        __mmask8 mask = ref_k1p_mask(m);
        GT(t1); int_k1p(ompNT, mask, m->chunkNum, m->val, m->col, m->chp, m->nmc, m->permi, vec, y); GT(t2);
        tt += measureTime(t2, t1);
      } break;
      case 4: {
        const str_matAXT *m = (const str_matAXT *)mat;
        fill_array(ompNT, m->nrows, 0, y);
        GT(t1); int_axt_noc_h1(ompNT, m->tileN, m->ax, m->sec, y); GT(t2);
        tt += measureTime(t2, t1);
      } break;
      case 5: {
        const str_matAXT *m = (const str_matAXT *)mat;
        fill_array(ompNT, m->nrows, 0, y);
        GT(t1); int_axt_noc(ompNT, m->tileN, m->tileH, m->ax, m->sec, y); GT(t2);
        tt += measureTime(t2, t1);
      } break;
      case 6: {
        const str_matAXT *m = (const str_matAXT *)mat;
        const UIN bn = ((m->tileN * HBRICK_SIZE) + bs - 1) / bs;
        fill_array(ompNT, m->nrows, 0, y);
        ref_shim_zero = 0;
        ref_shim_tracking = 1;
        GT(t1);
        int_axt_com_h1(ompNT, bn, bs, m->log, m->tileHW, m->tileN, m->lenAX, m->lenSEC, m->ax, m->sec, y);
        GT(t2);
        ref_shim_tracking = 0;
        ref_shim_zero = 1;
        ref_release_tracked();
        tt += measureTime(t2, t1);
      } break;
      default:
        return -1.0;
    }
  }
  if (ot) *ot = iters > 0 ? to / iters : 0.0;
  return iters > 0 ? tt / iters : 0.0;
}
