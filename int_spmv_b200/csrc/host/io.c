/*
 * io.c - matrix files and statistics of int_spmv_b200 (host side).
 *
 * File formats of the reference (intSpmv_main.c:187-249, "M:<line>"):
 *   .csr  text: "n nnz", then nnz lines "val col", then n+1 row pointers;
 *   .bin  binary: u32 n, u32 nnz, f64 val[nnz], u32 col[nnz], u32 row[n+1].
 * Unlike the reference, short reads and malformed headers are errors
 * (M:227-236 ignores fread counts) and the matrix is validated.
 *
 * printMatrixStats writes the reference's `.sta` report (M:286-300; same
 * lines and printf formats) next to the matrix file, replacing the extension
 * after the last '.' of the file name (the reference's strtok(name, ".")
 * truncates at the first '.' of the whole path, M:280-287).
 */
#define _GNU_SOURCE
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "intspmv.h"

#define API __attribute__((visibility("default")))

static int ends_with(const char *s, const char *suf) {
  const size_t a = strlen(s), b = strlen(suf);
  return a >= b && strcmp(s + a - b, suf) == 0;
}

API void ispmv_csr_free(str_matCSR *c) {
  if (!c) return;
  free(c->val); free(c->col); free(c->row); free(c->rl); free(c->rowStart); free(c->rowEnd);
  memset(c, 0, sizeof *c);
}

static int alloc_csr(str_matCSR *c, UIN n, UIN nnz) {
  memset(c, 0, sizeof *c);
  c->nrows = n;
  c->nnz = nnz;
  c->val = (FPT *)malloc((size_t)(nnz ? nnz : 1) * sizeof(FPT));
  c->col = (UIN *)malloc((size_t)(nnz ? nnz : 1) * sizeof(UIN));
  c->row = (UIN *)malloc(((size_t)n + 1) * sizeof(UIN));
  c->rl = (UIN *)calloc((size_t)n + 1, sizeof(UIN));
  if (!c->val || !c->col || !c->row || !c->rl) {
    ispmv_csr_free(c);
    return ISPMV_ERR_OOM;
  }
  return ISPMV_OK;
}

static int validate(const str_matCSR *c) {
  if (c->row[0] != 0 || c->row[c->nrows] != c->nnz) return ISPMV_ERR_ARG;
  for (UIN i = 0; i < c->nrows; i++)
    if (c->row[i + 1] < c->row[i]) return ISPMV_ERR_ARG;
  for (UIN j = 0; j < c->nnz; j++)
    if (c->col[j] >= c->nrows) return ISPMV_ERR_ARG;
  return ISPMV_OK;
}

API int ispmv_matrix_read(const char *path, str_matCSR *out) {
  if (!path || !out) return ISPMV_ERR_ARG;
  memset(out, 0, sizeof *out);
  const int txt = ends_with(path, ".csr"), bin = ends_with(path, ".bin");
  if (!txt && !bin) return ISPMV_ERR_ARG;
  FILE *fh = fopen(path, txt ? "r" : "rb");
  if (!fh) return ISPMV_ERR_ARG;
  int st = ISPMV_ERR_ARG;
  if (txt) {
    long long n, nnz;
    if (fscanf(fh, "%lld %lld", &n, &nnz) != 2 || n <= 0 || nnz < 0 || n >= 0xFFFFFFFFll ||
        nnz > 0xFFFFFFFFll)
      goto done;
    if ((st = alloc_csr(out, (UIN)n, (UIN)nnz)) != ISPMV_OK) goto done;
    st = ISPMV_ERR_ARG;
    for (long long i = 0; i < nnz; i++) {
      double v;
      long long c;
      if (fscanf(fh, "%lf %lld", &v, &c) != 2 || c < 0 || c >= n) goto fail;
      out->val[i] = v;
      out->col[i] = (UIN)c;
    }
    for (long long i = 0; i <= n; i++) {
      long long r;
      if (fscanf(fh, "%lld", &r) != 1 || r < 0 || r > nnz) goto fail;
      out->row[i] = (UIN)r;
    }
  } else {
    UIN hdr[2];
    if (fread(hdr, sizeof(UIN), 2, fh) != 2 || hdr[0] == 0 || hdr[0] == 0xFFFFFFFFu) goto done;
    if ((st = alloc_csr(out, hdr[0], hdr[1])) != ISPMV_OK) goto done;
    st = ISPMV_ERR_ARG;
    if (fread(out->val, sizeof(FPT), hdr[1], fh) != hdr[1]) goto fail;
    if (fread(out->col, sizeof(UIN), hdr[1], fh) != hdr[1]) goto fail;
    if (fread(out->row, sizeof(UIN), (size_t)hdr[0] + 1, fh) != (size_t)hdr[0] + 1) goto fail;
  }
  if ((st = validate(out)) != ISPMV_OK) goto fail;
  st = ISPMV_OK;
  goto done;
fail:
  ispmv_csr_free(out);
done:
  fclose(fh);
  return st;
}

API str_matCSR matrixReading(const char *matFileName) {
  str_matCSR c;
  const int st = ispmv_matrix_read(matFileName, &c);
  if (st != ISPMV_OK) {
    fflush(stdout);
    printf("\nmatrixReading is unable to read %s: %s\n\n", matFileName, ispmv_status_string(st));
    fflush(stdout);
    exit(EXIT_FAILURE);
  }
  return c;
}

API int ispmv_matrix_write(const char *path, const str_matCSR *c) {
  if (!path || !c || !c->row || c->nrows == 0) return ISPMV_ERR_ARG;
  const int txt = ends_with(path, ".csr"), bin = ends_with(path, ".bin");
  if (!txt && !bin) return ISPMV_ERR_ARG;
  FILE *fh = fopen(path, txt ? "w" : "wb");
  if (!fh) return ISPMV_ERR_ARG;
  int ok = 1;
  if (txt) {
    ok = fprintf(fh, "%u %u\n", c->nrows, c->nnz) > 0;
    for (UIN i = 0; ok && i < c->nnz; i++) ok = fprintf(fh, "%.17g %u\n", c->val[i], c->col[i]) > 0;
    for (UIN i = 0; ok && i <= c->nrows; i++) ok = fprintf(fh, "%u\n", c->row[i]) > 0;
  } else {
    const UIN hdr[2] = {c->nrows, c->nnz};
    ok = fwrite(hdr, sizeof(UIN), 2, fh) == 2 &&
         fwrite(c->val, sizeof(FPT), c->nnz, fh) == c->nnz &&
         fwrite(c->col, sizeof(UIN), c->nnz, fh) == c->nnz &&
         fwrite(c->row, sizeof(UIN), (size_t)c->nrows + 1, fh) == (size_t)c->nrows + 1;
  }
  if (fclose(fh) != 0) ok = 0;
  return ok ? ISPMV_OK : ISPMV_ERR_ARG;
}

API void printMatrixStats(const char *matFileName, str_matCSR *matCSR) {
  const int st = ispmv_csr_stats(matCSR);
  if (st != ISPMV_OK) {
    fflush(stdout);
    printf("\nprintMatrixStats: %s\n", ispmv_status_string(st));
    fflush(stdout);
    exit(EXIT_FAILURE);
  }
  const size_t L = strlen(matFileName);
  char *name = (char *)malloc(L + 8);
  if (!name) exit(EXIT_FAILURE);
  memcpy(name, matFileName, L + 1);
  char *slash = strrchr(name, '/');
  char *dot = strrchr(slash ? slash : name, '.');
  if (dot && dot != (slash ? slash + 1 : name)) *dot = '\0';
  strcat(name, ".sta");
  FILE *fh = fopen(name, "w+");
  free(name);
  if (!fh) return;
  const double rsdp = (matCSR->rsd / matCSR->rave) * 100;
  fprintf(fh, "------------------------------------\n");
  fprintf(fh, "matrix's statistics\n");
  fprintf(fh, "------------------------------------\n");
  fprintf(fh, "name:  %28s\n", matFileName);
  fprintf(fh, "nrows: %28d\n", matCSR->nrows);
  fprintf(fh, "nnz:   %28d\n", matCSR->nnz);
  fprintf(fh, "rmin:  %28d\n", matCSR->rmin);
  fprintf(fh, "rave:  %28.2lf\n", matCSR->rave);
  fprintf(fh, "rmax:  %28d\n", matCSR->rmax);
  fprintf(fh, "rsd:   %28.2lf\n", matCSR->rsd);
  fprintf(fh, "rsdp:  %28.2lf\n", rsdp);
  fprintf(fh, "bw:    %28d\n", matCSR->bw);
  fclose(fh);
}
