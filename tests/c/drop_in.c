/*
 * drop_in.c - the reference's driver (intSpmv_main.c:1617-1761) written
 * against include/intspmv.h and linked with libintspmv.so, as a caller of
 * the reference would: read the matrix, print its statistics, build every
 * format with the reference-named builders, time every kernel through the
 * test_* harness and print the reference's two tables.  Built twice by
 * tests/test_c_drop_in.py: FP_TYPE=FP_DOUBLE (the default) and
 * FP_TYPE=FP_FLOAT (FPT = float, the `_f32` symbols).
 *
 *   drop_in <matrix.csr|.bin> <outdir>
 *
 * Besides the tables, y of every kernel (one call of each reference-named
 * kernel, with the reference's zeroed y for the AXT kernels) is written to
 * <outdir>/<kernel>.y as raw FPT, for the test to check against the oracle.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "intspmv.h"

static void dump(const char *dir, const char *name, const FPT *y, UIN n) {
  char path[512];
  snprintf(path, sizeof path, "%s/%s.y", dir, name);
  FILE *f = fopen(path, "wb");
  if (!f || fwrite(y, sizeof(FPT), n, f) != n) {
    printf("cannot write %s\n", path);
    exit(EXIT_FAILURE);
  }
  fclose(f);
}

static void row(const str_res *r) {
  printf("%25s %15.7lf %8.3lf %15.7lf %11.3le %13.3le %12d\n", r->name, r->et, r->flops * 1e-9, r->ot,
         r->sErr.aErr, r->sErr.rErr, (int)r->sErr.pos);
}

int main(int argc, char **argv) {
  if (argc < 3) {
    printf("usage: %s <matrix.csr|.bin> <outdir>\n", argv[0]);
    return EXIT_FAILURE;
  }
  printf("FPT: %s (%zu bytes)\n", sizeof(FPT) == 4 ? "float" : "double", sizeof(FPT));
  str_matCSR csr = matrixReading(argv[1]);
  printMatrixStats(argv[1], &csr);
  str_formatData fd[16];
  int nfd = 0;
  fd[nfd++] = getFormatDataCSR(&csr);
  const UIN n = csr.nrows;
  FPT *vr = (FPT *)calloc(n, sizeof(FPT));
  FPT *yr = (FPT *)calloc(n, sizeof(FPT));
  FPT *y = (FPT *)calloc(n + 1, sizeof(FPT));
  initVec(n, vr);
  cf_CSR(csr, vr, yr);
  dump(argv[2], "cf_CSR", yr, n);
  str_res sr[16];
  int nsr = 0;
  sr[nsr++] = test_cf_CSR(csr, vr, yr);

  str_matAXC axc;
  fd[nfd++] = getFormatDataAXC(0, csr, vr, &axc);
  sr[nsr++] = test_int_AXC(0, axc, yr);
  int_axc(0, n, axc.ax, axc.brp, y);
  dump(argv[2], "int_axc", y, n);

  str_matK1 k1;
  fd[nfd++] = getFormatDataK1(ISPMV_CHUNK_SIZE, csr, vr, &k1);
  sr[nsr++] = test_int_k1(0, k1, vr, yr);
  sr[nsr++] = test_int_k1p(0, k1, vr, yr);
  FPT *res = (FPT *)calloc((size_t)k1.chunkNum * ISPMV_CHUNK_SIZE + 1, sizeof(FPT));
  int_k1(0, k1.chunkNum, k1.val, k1.col, k1.chp, k1.nmc, vr, res);
  memset(y, 0, (size_t)n * sizeof(FPT));
  orderArrayK1(0, n, k1.permi, res, y);
  dump(argv[2], "int_k1", y, n);
  {
    const UIN pad = k1.chunkNum * ISPMV_CHUNK_SIZE - n; /* the tail mask, M:1076-1086 */
    const unsigned char mask = (unsigned char)(0xFFu >> pad);
    memset(y, 0, (size_t)(n + 1) * sizeof(FPT));
    int_k1p(0, mask, k1.chunkNum, k1.val, k1.col, k1.chp, k1.nmc, k1.permi, vr, y);
    dump(argv[2], "int_k1p", y, n);
  }
  free(res);

  static const struct { UIN bs, th; const char *mode; } axt[] = {
      {128, 1, "NOC"}, {128, 4, "NOC"}, {128, 8, "NOC"}, {128, 1, "COM"}, {256, 1, "COM"}, {512, 1, "COM"}};
  for (int a = 0; a < 6; a++) {
    str_matAXT m;
    fd[nfd++] = getFormatDataAXT(0, axt[a].bs, 8, axt[a].th, axt[a].mode, csr, vr, &m);
    memset(y, 0, (size_t)n * sizeof(FPT)); /* AXT kernels accumulate: y zeroed, M:1421 */
    if (strcmp(axt[a].mode, "COM") == 0) {
      sr[nsr++] = test_int_axt_com_h1(0, axt[a].bs, m, yr);
      const UIN bn = (m.tileN * ISPMV_HBRICK_SIZE + axt[a].bs - 1) / axt[a].bs;
      int_axt_com_h1(0, bn, axt[a].bs, m.log, m.tileHW, m.tileN, m.lenAX, m.lenSEC, m.ax, m.sec, y);
    } else if (axt[a].th == 1) {
      sr[nsr++] = test_int_axt_noc_h1(0, m, yr);
      int_axt_noc_h1(0, m.tileN, m.ax, m.sec, y);
    } else {
      sr[nsr++] = test_int_axt_noc(0, m, yr);
      int_axt_noc(0, m.tileN, m.tileH, m.ax, m.sec, y);
    }
    dump(argv[2], sr[nsr - 1].name, y, n);
    ispmv_free_axt(&m);
  }

  printf("formats' data\n");
  printf("%22s %20s %10s %20s\n", "format", "memory [Mbytes]", "occupancy", "convTime [s]");
  for (int i = 0; i < nfd; i++)
    printf("%22s %20.2lf %10.2lf %20.6lf\n", fd[i].name, fd[i].mfp * 1e-6, fd[i].beta, fd[i].ct);
  printf("kernels' results\n");
  printf("%25s %15s %8s %15s %13s %13s %10s\n", "kernel", "exeTime [s]", "Gflops", "ordTime [s]", "aErr||.||inf",
         "rErr||.||inf", "rowInd");
  for (int i = 0; i < nsr; i++) row(&sr[i]);

  ispmv_free_axc(&axc);
  ispmv_free_k1(&k1);
  free(vr);
  free(yr);
  free(y);
  ispmv_csr_free(&csr);
  return EXIT_SUCCESS;
}
