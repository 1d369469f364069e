/*
 * builders.c - host format builders of int_spmv_b200.
 *
 * Each builder produces, for a CSR matrix with row lengths filled, the
 * arrays of one reference format (edoardoCB/int_spmv, intSpmv_main.c; cited
 * M:<line>), bit-exact to the reference's: AXC brp/ax, K1 permi/nmc/chp/
 * val/col, AXT con/sec/ax.  The layouts are computed here in closed form
 * from a per-row prefix of slot counts, in parallel over rows, instead of the
 * reference's incremental pointer walks; the rules that must match are:
 *
 *   AXC (M:619-658):  brp[r+1] = brp[r] + 16*ceil(rl/8); element k of row r
 *       at ax[brp[r] + 16*(k/8) + k%8], its x copy at +8.
 *   K1 (M:775-837):   rows by length descending, equal lengths by ascending
 *       id; chunk c of 8 rows holds nmc[c] = its first row's length columns,
 *       column-major: val[chp[c] + 8*k + lane].
 *   AXT (M:1118-1260): a running slot count s over rows (each row padded to
 *       a multiple of 8 (tileH=1) or tileH (tileH>1) in NOC mode, packed in
 *       COM mode).  Slot s lives in tile T = s/(8*th), column C = (s/th)%8,
 *       sub-row R = s%th, i.e. at ax[T*16*th + R*16 + C] (value) and +8 (x).
 *       con[r] is that position for the row's first slot.  sec is the row of
 *       each tile (NOC, th=1), of each tile column (NOC, th>1), or a segment
 *       descriptor (row << log2 bs) | min(left-1, bs-1-s%bs) at each row
 *       start and block start (COM).
 * Padding of every array is zero (the reference zero-fills AXT, M:1304-1305,
 * and relies on fresh pages for AXC/K1).
 *
 * Allocation contract (M:668,684,847-849,877-878,1284,1302-1303): arrays are
 * allocated inside the struct - index arrays with calloc/malloc, value arrays
 * 64-byte aligned - and the caller releases every one with free().
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "intspmv.h"

#define API __attribute__((visibility("default")))
#define HBW ISPMV_HBRICK_SIZE
#define CHK ISPMV_CHUNK_SIZE

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static int nthreads(UIN ompNT) {
#ifdef _OPENMP
  return ompNT ? (int)ompNT : omp_get_max_threads();
#else
  (void)ompNT;
  return 1;
#endif
}

/* 64-byte aligned, zeroed, at least one element (callers free()). */
static void *alloc64z(size_t bytes) {
  void *p = NULL;
  if (bytes == 0) bytes = 64;
  bytes = (bytes + 63) & ~(size_t)63;
  if (posix_memalign(&p, 64, bytes) != 0) return NULL;
  memset(p, 0, bytes);
  return p;
}

static void *callocz(size_t n, size_t sz) { return calloc(n ? n : 1, sz); }

/* ------------------------------------------------------------------------ */
API int ispmv_csr_stats(str_matCSR *csr) {
  if (!csr || !csr->row || !csr->rl || csr->nrows == 0) return ISPMV_ERR_ARG;
  if (csr->nnz && (!csr->col || !csr->val)) return ISPMV_ERR_ARG;
  const UIN n = csr->nrows;
  if (csr->row[0] != 0 || csr->row[n] != csr->nnz) return ISPMV_ERR_ARG;
  UIN mn = 1000000000u, mx = 0, bw = 0;
  double s1 = 0.0, s2 = 0.0;
  int bad = 0;
  for (UIN i = 0; i < n; i++) {
    if (csr->row[i + 1] < csr->row[i]) { bad = 1; break; }
    const UIN l = csr->row[i + 1] - csr->row[i];
    csr->rl[i] = l;
    s1 += l;
    s2 += (double)(l * l); /* u32 product, as M:264 */
    mn = mn < l ? mn : l;
    mx = mx > l ? mx : l;
  }
  if (bad) return ISPMV_ERR_ARG;
  const UIN nnz = csr->nnz;
#pragma omp parallel for reduction(max : bw) reduction(|| : bad) schedule(static)
  for (UIN i = 0; i < n; i++) {
    for (UIN j = csr->row[i]; j < csr->row[i + 1]; j++) {
      const UIN c = csr->col[j];
      if (c >= n) bad = 1;
      const int d = abs((int)i - (int)c);
      bw = ((UIN)d > bw) ? (UIN)d : bw;
    }
  }
  (void)nnz;
  if (bad) return ISPMV_ERR_ARG;
  s1 /= (double)n;
  s2 /= (double)n;
  csr->rmin = mn;
  csr->rave = s1;
  csr->rmax = mx;
  csr->rsd = sqrt(s2 - s1 * s1);
  csr->bw = bw;
  return ISPMV_OK;
}

/* Exclusive prefix of per-row counts (u64), parallel two-pass. */
static void prefix_u64(UIN n, const uint64_t *cnt, uint64_t *off, int nt) {
  if (nt < 2 || n < 65536) {
    uint64_t s = 0;
    for (UIN i = 0; i < n; i++) { off[i] = s; s += cnt[i]; }
    off[n] = s;
    return;
  }
  uint64_t *part = (uint64_t *)calloc((size_t)nt + 1, sizeof(uint64_t));
  if (!part) { /* fall back to serial */
    uint64_t s = 0;
    for (UIN i = 0; i < n; i++) { off[i] = s; s += cnt[i]; }
    off[n] = s;
    return;
  }
#pragma omp parallel num_threads(nt)
  {
#ifdef _OPENMP
    const int t = omp_get_thread_num(), T = omp_get_num_threads();
#else
    const int t = 0, T = 1;
#endif
    const UIN lo = (UIN)(((uint64_t)n * t) / T), hi = (UIN)(((uint64_t)n * (t + 1)) / T);
    uint64_t s = 0;
    for (UIN i = lo; i < hi; i++) s += cnt[i];
    part[t + 1] = s;
#pragma omp barrier
#pragma omp single
    for (int k = 1; k <= T; k++) part[k] += part[k - 1];
    s = part[t];
    for (UIN i = lo; i < hi; i++) { off[i] = s; s += cnt[i]; }
    if (t == T - 1) off[n] = s;
  }
  free(part);
}

static void set_format_data(str_formatData *fd, const char *name, double mfp, double beta, double ct) {
  if (!fd) return;
  memset(fd->name, 0, sizeof fd->name);
  snprintf(fd->name, sizeof fd->name, "%s", name);
  fd->mfp = mfp;
  fd->beta = beta;
  fd->ct = ct;
}

/* ---------------------------------------------------------------- CSR -- */
/* getFormatDataCSR, M:324-357 */
API int ispmv_build_csr(str_matCSR *csr, str_formatData *fd) {
  if (!csr || !csr->row || csr->nrows == 0) return ISPMV_ERR_ARG;
  const double t0 = now_s();
  const UIN n = csr->nrows;
  UIN *rs = (UIN *)callocz(n, sizeof(UIN)), *re = (UIN *)callocz(n, sizeof(UIN));
  if (!rs || !re) { free(rs); free(re); return ISPMV_ERR_OOM; }
  for (UIN i = 0; i < n; i++) { rs[i] = csr->row[i]; re[i] = csr->row[i + 1]; }
  csr->rowStart = rs;
  csr->rowEnd = re;
  const double mfp = (double)csr->nnz * sizeof(FPT) + (double)csr->nnz * sizeof(UIN) +
                     (double)(n + 1) * sizeof(UIN) + (double)n * sizeof(FPT);
  set_format_data(fd, "CSR", mfp, 1.0, now_s() - t0);
  return ISPMV_OK;
}

/* ---------------------------------------------------------------- AXC -- */
API int ispmv_build_axc(UIN ompNT, const str_matCSR *csr, const FPT *vec, str_matAXC *m,
                        str_formatData *fd) {
  if (!csr || !m || !vec || !csr->rl || !csr->row || csr->nrows == 0) return ISPMV_ERR_ARG;
  const double t0 = now_s();
  const UIN n = csr->nrows;
  const int nt = nthreads(ompNT);
  memset(m, 0, sizeof *m);
  m->nrows = n;
  m->nnz = csr->nnz;
  m->lenBRP = n + 1;
  uint64_t *cnt = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
  uint64_t *off = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
  if (!cnt || !off) { free(cnt); free(off); return ISPMV_ERR_OOM; }
#pragma omp parallel for num_threads(nt) schedule(static)
  for (UIN r = 0; r < n; r++) cnt[r] = 2ull * HBW * ((csr->rl[r] + HBW - 1) / HBW);
  prefix_u64(n, cnt, off, nt);
  free(cnt);
  if (off[n] > 0xFFFFFFFFull) { free(off); return ISPMV_ERR_OVERFLOW; }
  m->brp = (UIN *)callocz((size_t)n + 1, sizeof(UIN));
  if (!m->brp) { free(off); return ISPMV_ERR_OOM; }
#pragma omp parallel for num_threads(nt) schedule(static)
  for (UIN r = 0; r <= n; r++) m->brp[r] = (UIN)off[r];
  free(off);
  m->lenAX = m->brp[n];
  m->ax = (FPT *)alloc64z((size_t)m->lenAX * sizeof(FPT));
  if (!m->ax) { free(m->brp); m->brp = NULL; return ISPMV_ERR_OOM; }
  const UIN *row = csr->row, *col = csr->col;
  const FPT *val = csr->val;
  FPT *ax = m->ax;
  const UIN *brp = m->brp;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
  for (UIN r = 0; r < n; r++) {
    const UIN b = brp[r], j0 = row[r];
    for (UIN j = j0; j < row[r + 1]; j++) {
      const UIN k = j - j0;
      const size_t p = (size_t)b + 2 * HBW * (k / HBW) + k % HBW;
      ax[p] = val[j];
      ax[p + HBW] = vec[col[j]];
    }
  }
  const double mfp = (double)m->lenAX * sizeof(FPT) + (double)m->lenBRP * sizeof(UIN);
  const double beta = m->lenAX ? (double)m->nnz / (double)(m->lenAX >> 1) : 0.0;
  set_format_data(fd, "AXC", mfp, beta, now_s() - t0);
  return ISPMV_OK;
}

API int ispmv_build_axc_cols(UIN ompNT, const str_matCSR *csr, const str_matAXC *m, UIN **axi) {
  if (!csr || !m || !axi || !m->brp || m->nrows != csr->nrows) return ISPMV_ERR_ARG;
  const int nt = nthreads(ompNT);
  UIN *c = (UIN *)callocz((size_t)m->lenAX / 2, sizeof(UIN));
  if (!c) return ISPMV_ERR_OOM;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
  for (UIN r = 0; r < m->nrows; r++) {
    const size_t v0 = m->brp[r] / 2;
    for (UIN j = csr->row[r]; j < csr->row[r + 1]; j++) c[v0 + (j - csr->row[r])] = csr->col[j];
  }
  *axi = c;
  return ISPMV_OK;
}

/* ----------------------------------------------------------------- K1 -- */
API int ispmv_build_k1(UIN blockSize, const str_matCSR *csr, const FPT *vec, str_matK1 *m,
                       str_formatData *fd) {
  (void)blockSize; /* unused by the reference too (M:841) */
  (void)vec;       /* K1 gathers x at kernel time (M:957) */
  if (!csr || !m || !csr->rl || !csr->row || csr->nrows == 0) return ISPMV_ERR_ARG;
  const double t0 = now_s();
  const UIN n = csr->nrows;
  memset(m, 0, sizeof *m);
  m->nrows = n;
  m->nnz = csr->nnz;
  m->chunkNum = (n + CHK - 1) / CHK;
  const UIN cn = m->chunkNum;
  m->permi = (UIN *)alloc64z(((size_t)cn + 1) * CHK * sizeof(UIN));
  m->nmc = (UIN *)callocz(cn, sizeof(UIN));
  m->chp = (UIN *)callocz(cn, sizeof(UIN));
  if (!m->permi || !m->nmc || !m->chp) goto oom;
  {
    /* Stable counting sort by length, descending: equal lengths keep the
     * ascending row order the reference's (stable) qsort gives. */
    UIN maxl = 0;
    for (UIN r = 0; r < n; r++) maxl = csr->rl[r] > maxl ? csr->rl[r] : maxl;
    size_t *bucket = (size_t *)calloc((size_t)maxl + 2, sizeof(size_t));
    if (!bucket) goto oom;
    for (UIN r = 0; r < n; r++) bucket[maxl - csr->rl[r] + 1]++;
    for (size_t b = 1; b <= (size_t)maxl + 1; b++) bucket[b] += bucket[b - 1];
    for (UIN r = 0; r < n; r++) m->permi[bucket[maxl - csr->rl[r]]++] = r;
    free(bucket);
  }
  {
    uint64_t len = 0;
    for (UIN c = 0; c < cn; c++) {
      m->nmc[c] = csr->rl[m->permi[(size_t)c * CHK]];
      m->chp[c] = (UIN)len;
      len += (uint64_t)CHK * m->nmc[c];
      if (len > 0xFFFFFFFFull) {
        free(m->permi); free(m->nmc); free(m->chp);
        memset(m, 0, sizeof *m);
        return ISPMV_ERR_OVERFLOW;
      }
    }
    m->lenVC = (UIN)len;
  }
  m->val = (FPT *)alloc64z((size_t)m->lenVC * sizeof(FPT));
  m->col = (UIN *)alloc64z((size_t)m->lenVC * sizeof(UIN));
  if (!m->val || !m->col) goto oom;
#pragma omp parallel for schedule(dynamic, 256)
  for (UIN c = 0; c < cn; c++) {
    for (UIN lane = 0; lane < CHK; lane++) {
      const size_t i = (size_t)c * CHK + lane;
      if (i >= n) break;
      const UIN r = m->permi[i], j0 = csr->row[r];
      for (UIN j = j0; j < csr->row[r + 1]; j++) {
        const size_t p = (size_t)m->chp[c] + (size_t)(j - j0) * CHK + lane;
        m->val[p] = csr->val[j];
        m->col[p] = csr->col[j];
      }
    }
  }
  {
    const double mfp = 2.0 * cn * sizeof(UIN) + (double)m->lenVC * (sizeof(FPT) + sizeof(UIN)) +
                       (double)n * sizeof(UIN) + (double)n * sizeof(FPT);
    const double beta = m->lenVC ? (double)m->nnz / (double)m->lenVC : 0.0;
    set_format_data(fd, "K1", mfp, beta, now_s() - t0);
  }
  return ISPMV_OK;
oom:
  free(m->permi); free(m->nmc); free(m->chp); free(m->val); free(m->col);
  memset(m, 0, sizeof *m);
  return ISPMV_ERR_OOM;
}

/* ---------------------------------------------------------------- AXT -- */
static UIN floor_log2_lt1024(UIN v) {
  /* M:1286-1287 / M:1341-1348: the largest i < 10 with (v >> i) == 1 */
  UIN r = 0;
  for (UIN i = 0; i < 10; i++)
    if ((v >> i) == 1) r = i;
  return r;
}

/* position in ax of slot s (value half) */
static inline size_t axt_pos(uint64_t s, UIN thw, UIN th) {
  const uint64_t ths = (uint64_t)thw * th;
  const uint64_t T = s / ths, w = s % ths;
  return (size_t)(T * 2 * ths + (w % th) * 2 * thw + w / th);
}

API int ispmv_build_axt(UIN ompNT, UIN bs, UIN thw, UIN th, const char *mode, const str_matCSR *csr,
                        const FPT *vec, str_matAXT *m, str_formatData *fd) {
  if (!csr || !m || !vec || !mode || !csr->rl || !csr->row || csr->nrows == 0) return ISPMV_ERR_ARG;
  if (thw == 0 || th == 0) return ISPMV_ERR_ARG;
  const int noc = strcmp(mode, "NOC") == 0, com = strcmp(mode, "COM") == 0;
  if (!noc && !com) return ISPMV_ERR_ARG;
  if (com && th != 1) return ISPMV_ERR_UNSUPPORTED; /* unimplemented in the reference, M:1338-1362 */
  UIN lg = 0;
  if (com) {
    if (bs < 2 || bs > 512 || (bs & (bs - 1))) return ISPMV_ERR_ARG;
    lg = floor_log2_lt1024(bs);
    if (((uint64_t)(csr->nrows - 1) << lg) > 0xFFFFFFFFull) return ISPMV_ERR_OVERFLOW; /* row << log */
  }
  const double t0 = now_s();
  const UIN n = csr->nrows;
  const int nt = nthreads(ompNT);
  const UIN grp = (th == 1) ? thw : th;
  memset(m, 0, sizeof *m);
  m->nrows = n;
  m->nnz = csr->nnz;
  snprintf(m->mode, sizeof m->mode, "%s", mode);
  m->tileHW = thw;
  m->tileH = th;
  m->logTH = floor_log2_lt1024(th);
  m->lenCON = n;
  m->log = lg;

  uint64_t *cnt = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
  uint64_t *off = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
  if (!cnt || !off) { free(cnt); free(off); return ISPMV_ERR_OOM; }
#pragma omp parallel for num_threads(nt) schedule(static)
  for (UIN r = 0; r < n; r++) {
    const uint64_t l = csr->rl[r];
    cnt[r] = noc ? ((l + grp - 1) / grp) * grp : l;
  }
  prefix_u64(n, cnt, off, nt);
  free(cnt);
  /* Total tile columns: every row's slot count is a multiple of th in NOC
   * mode and th == 1 in COM mode, so columns = slots / th. */
  const uint64_t slots = off[n], columns = slots / th;
  const uint64_t tiles = (columns + thw - 1) / thw;
  const uint64_t lenAX = tiles * 2 * thw * th;
  const uint64_t lenSEC = (noc && th == 1) ? tiles : (noc ? tiles * thw : tiles * thw * th);
  if (lenAX > 0xFFFFFFFFull || lenSEC > 0xFFFFFFFFull) { free(off); return ISPMV_ERR_OVERFLOW; }
  m->tileN = (UIN)tiles;
  m->lenAX = (UIN)lenAX;
  m->lenSEC = (UIN)lenSEC;
  m->con = (UIN *)callocz(n, sizeof(UIN));
  m->ax = (FPT *)alloc64z((size_t)lenAX * sizeof(FPT));
  m->sec = (UIN *)alloc64z((size_t)lenSEC * sizeof(UIN));
  if (!m->con || !m->ax || !m->sec) {
    free(off); free(m->con); free(m->ax); free(m->sec);
    memset(m, 0, sizeof *m);
    return ISPMV_ERR_OOM;
  }
  const UIN *row = csr->row, *col = csr->col;
  const FPT *val = csr->val;
  FPT *ax = m->ax;
  UIN *sec = m->sec;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
  for (UIN r = 0; r < n; r++) {
    const uint64_t s0 = off[r];
    m->con[r] = (UIN)axt_pos(s0, thw, th);
    const UIN j0 = row[r], len = row[r + 1] - j0;
    for (UIN k = 0; k < len; k++) {
      const uint64_t s = s0 + k;
      const size_t p = axt_pos(s, thw, th);
      ax[p] = val[j0 + k];
      ax[p + thw] = vec[col[j0 + k]];
      if (noc) {
        const uint64_t T = s / ((uint64_t)thw * th);
        sec[th == 1 ? T : T * thw + (s / th) % thw] = r;
      } else if (k == 0 || s % bs == 0) {
        const UIN q1 = len - k - 1, q2 = bs - 1 - (UIN)(s % bs);
        sec[s] = (r << lg) | (q1 > q2 ? q2 : q1);
      }
    }
  }
  free(off);
  char name[24];
  if (noc && th == 1) snprintf(name, sizeof name, "AXT_NOC_H1_HW8");
  else if (noc) snprintf(name, sizeof name, "AXT_NOC_H%u_HW8", th);
  else snprintf(name, sizeof name, "AXT_COM_H1_HW8_BS%u", bs);
  const double mfp = (double)m->lenAX * sizeof(FPT) + (double)m->lenSEC * sizeof(UIN);
  const double beta = m->lenAX ? (double)m->nnz / (double)(m->lenAX >> 1) : 0.0;
  set_format_data(fd, name, mfp, beta, now_s() - t0);
  return ISPMV_OK;
}

/* Slot of the first element of row r, recovered from con[r] (inverse of axt_pos). */
static inline uint64_t axt_slot_of_con(UIN con, UIN thw, UIN th) {
  const uint64_t ths = (uint64_t)thw * th, two = 2 * ths;
  const uint64_t T = con / two, rem = con % two;
  const uint64_t R = rem / (2 * thw), C = rem % (2 * thw);
  return T * ths + C * th + R;
}

API int ispmv_build_axt_cols(UIN ompNT, const str_matCSR *csr, const str_matAXT *m, UIN **axi) {
  if (!csr || !m || !axi || !m->con || m->nrows != csr->nrows || m->tileHW == 0 || m->tileH == 0)
    return ISPMV_ERR_ARG;
  const int nt = nthreads(ompNT);
  const UIN thw = m->tileHW, th = m->tileH;
  UIN *c = (UIN *)alloc64z((size_t)m->lenAX / 2 * sizeof(UIN));
  if (!c) return ISPMV_ERR_OOM;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
  for (UIN r = 0; r < m->nrows; r++) {
    const UIN j0 = csr->row[r], len = csr->row[r + 1] - j0;
    if (!len) continue;
    const uint64_t s0 = axt_slot_of_con(m->con[r], thw, th);
    for (UIN k = 0; k < len; k++) {
      const size_t p = axt_pos(s0 + k, thw, th);
      c[(p / (2 * thw)) * thw + p % (2 * thw)] = csr->col[j0 + k];
    }
  }
  *axi = c;
  return ISPMV_OK;
}

API void ispmv_free_axc(str_matAXC *m) {
  if (!m) return;
  free(m->ax);
  free(m->brp);
  memset(m, 0, sizeof *m);
}
API void ispmv_free_k1(str_matK1 *m) {
  if (!m) return;
  free(m->permi); free(m->nmc); free(m->chp); free(m->val); free(m->col);
  memset(m, 0, sizeof *m);
}
API void ispmv_free_axt(str_matAXT *m) {
  if (!m) return;
  free(m->ax); free(m->sec); free(m->con);
  memset(m, 0, sizeof *m);
}

/* ------------------------------------------------- errors and x ramp -- */
API void getErrors(const UIN len, const FPT *ar, const FPT *ac, str_err *e) {
  double maxDif = 0.0, maxVal = 0.0;
  UIN pos = 0;
  for (UIN i = 0; i < len; i++) {
    const double v = fabs(ar[i]);
    if (v > maxVal) maxVal = v;
    const double d = fabs(fabs(ac[i]) - v);
    if (d > maxDif) { maxDif = d; pos = i; }
  }
  e->aErr = maxDif;
  e->rErr = maxDif / maxVal;
  e->pos = pos;
}

API void initVec(const UIN len, FPT *vec) {
  for (UIN i = 0; i < len; i++) vec[i] = (FPT)i;
}

/* fill_array, M:371-378: array[i] = val on ompNT threads (0: all). */
API void fill_array(const UIN ompNT, const UIN len, FPT val, FPT *array) {
  const int nt = nthreads(ompNT);
#pragma omp parallel for num_threads(nt) schedule(static)
  for (long long i = 0; i < (long long)len; i++) array[i] = val;
}

/* --------------------------------------- compat (exit-on-error) forms -- */
static void die(const char *fn, int st) {
  fflush(stdout);
  printf("\n%s failed: %s\n", fn, ispmv_status_string(st));
  fflush(stdout);
  exit(EXIT_FAILURE);
}

API str_formatData getFormatDataCSR(str_matCSR *matCSR) {
  str_formatData fd;
  const int st = ispmv_build_csr(matCSR, &fd);
  if (st) die("getFormatDataCSR", st);
  return fd;
}
API str_formatData getFormatDataAXC(const UIN ompNumThreads, const str_matCSR matCSR, const FPT *vec,
                                    str_matAXC *matAXC) {
  str_formatData fd;
  const int st = ispmv_build_axc(ompNumThreads, &matCSR, vec, matAXC, &fd);
  if (st) die("getFormatDataAXC", st);
  return fd;
}
API str_formatData getFormatDataK1(const UIN blockSize, const str_matCSR matCSR, const FPT *vec,
                                   str_matK1 *matK1) {
  str_formatData fd;
  const int st = ispmv_build_k1(blockSize, &matCSR, vec, matK1, &fd);
  if (st) die("getFormatDataK1", st);
  return fd;
}
API str_formatData getFormatDataAXT(const UIN ompNT, const UIN bs, const UIN thw, const UIN th,
                                    const char *mode, const str_matCSR matCSR, const FPT *vec,
                                    str_matAXT *matAXT) {
  str_formatData fd;
  const int st = ispmv_build_axt(ompNT, bs, thw, th, mode, &matCSR, vec, matAXT, &fd);
  if (st) die("getFormatDataAXT", st);
  return fd;
}

#ifndef ISPMV_FPT_FLOAT /* the batched path is FP64 */
/* ------------------------------------------------- batched matrices -- */
/* Block-diagonal CSR of `count` square matrices: matrix m's rows and columns
 * start at off[m] (off has count+1 entries).  Arrays are malloc'd (free with
 * ispmv_csr_free); rl and the statistics are filled. */
API int ispmv_csr_blockdiag(UIN count, const str_matCSR *mats, str_matCSR *out, UIN *off) {
  if (!mats || !out || !off || count == 0) return ISPMV_ERR_ARG;
  uint64_t n = 0, nnz = 0;
  for (UIN m = 0; m < count; m++) {
    if (!mats[m].row || mats[m].nrows == 0) return ISPMV_ERR_ARG;
    off[m] = (UIN)n;
    n += mats[m].nrows;
    nnz += mats[m].row[mats[m].nrows];
    if (n >= 0xFFFFFFFFull || nnz > 0xFFFFFFFFull) return ISPMV_ERR_OVERFLOW;
  }
  off[count] = (UIN)n;
  memset(out, 0, sizeof *out);
  out->nrows = (UIN)n;
  out->nnz = (UIN)nnz;
  out->row = (UIN *)malloc(((size_t)n + 1) * sizeof(UIN));
  out->rl = (UIN *)calloc((size_t)n + 1, sizeof(UIN));
  out->col = (UIN *)malloc((size_t)(nnz ? nnz : 1) * sizeof(UIN));
  out->val = (FPT *)malloc((size_t)(nnz ? nnz : 1) * sizeof(FPT));
  if (!out->row || !out->rl || !out->col || !out->val) {
    free(out->row); free(out->rl); free(out->col); free(out->val);
    memset(out, 0, sizeof *out);
    return ISPMV_ERR_OOM;
  }
  uint64_t j = 0;
  out->row[0] = 0;
  for (UIN m = 0; m < count; m++) {
    const str_matCSR *a = &mats[m];
    const UIN base = off[m], an = a->nrows, annz = a->row[an];
    for (UIN r = 0; r < an; r++) out->row[base + r + 1] = (UIN)j + a->row[r + 1];
    for (UIN q = 0; q < annz; q++) {
      if (a->col[q] >= an) { free(out->row); free(out->rl); free(out->col); free(out->val);
        memset(out, 0, sizeof *out); return ISPMV_ERR_ARG; }
      out->col[j + q] = a->col[q] + base;
      out->val[j + q] = a->val[q];
    }
    j += annz;
  }
  return ispmv_csr_stats(out);
}
#endif
