/*
 * oracle.c - TEST INFRASTRUCTURE ONLY.  A plain-C, single-threaded
 * restatement of the reference's (edoardoCB/int_spmv, intSpmv_main.c)
 * algorithms on the SpMV path: row statistics, the AXC / K1 / AXT format
 * builders, the naive CSR product, the reference's CPU kernels and its error
 * metric.  Every function cites the reference lines it restates (M:<line> =
 * intSpmv_main.c:<line>).
 *
 * Only tests, the smoke check and the CPU-baseline leg of bench.py use this
 * file, and only as the checker; the product (int_spmv_b200) never links or
 * calls it.  It is pinned against the reference itself, compiled from its own
 * source by oracle/Makefile into oracle/_ref (tests/test_oracle_pin.py), and
 * against the golden fixtures that reference build generated (tests/golden/).
 *
 * Arithmetic follows the reference as GCC compiles it with -O3 -mavx512f
 * (the scalar CSR loop and int_axt_noc's lane sums unfused, the 8-lane
 * accumulations of int_k1 / int_k1p contracted to FMA, GCC's
 * _mm512_reduce_add_pd tree), so the deterministic kernels agree with the reference bit for bit
 * (checked by tests/test_oracle_pin.py).  Build with -ffp-contract=off:
 * every fused operation below is an explicit fma().
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double FPT;
typedef unsigned int UIN;

#define ORC_API __attribute__((visibility("default")))
#define HBW 8u /* HBRICK_SIZE, M:101-103 */
#define CHK 8u /* CHUNK_SIZE, M:107-109 */

/* GCC's _mm512_reduce_add_pd on lanes a[0..7]: halves, then quarters, then
 * the last pair (used by int_axc M:726 and int_axt_noc_h1 M:1398). */
static FPT orc_reduce8(const FPT *a) {
  FPT t3[4], t6[2];
  for (int i = 0; i < 4; i++) t3[i] = a[4 + i] + a[i];
  for (int j = 0; j < 2; j++) t6[j] = t3[2 + j] + t3[j];
  return t6[0] + t6[1];
}

/* ---- M:253-278: row lengths and statistics (printMatrixStats without the file) ---- */
ORC_API void orc_stats(UIN n, const UIN *row, const UIN *col, UIN *rl, UIN *rmin, double *rave,
                       UIN *rmax, double *rsd, UIN *bw) {
  UIN mn = 1000000000u, mx = 0, b = 0;
  double s1 = 0.0, s2 = 0.0;
  for (UIN i = 0; i < n; i++) {
    UIN l = row[i + 1] - row[i];
    rl[i] = l;
    s1 += l;
    s2 += (double)(l * l); /* M:264: rl*rl is a u32 product */
    mn = mn < l ? mn : l;
    mx = mx > l ? mx : l;
    for (UIN j = row[i]; j < row[i + 1]; j++) {
      int d = abs((int)i - (int)col[j]);
      b = ((UIN)d > b) ? (UIN)d : b; /* M:269: dif > bw compares int with UIN */
    }
  }
  s1 /= (double)n;
  s2 /= (double)n;
  *rmin = mn;
  *rave = s1;
  *rmax = mx;
  *rsd = sqrt(s2 - s1 * s1);
  *bw = b;
}

/* ---- M:382-396: the naive CSR product (the oracle y) ---- */
ORC_API void orc_cf_csr(UIN n, const UIN *row, const UIN *col, const FPT *val, const FPT *x, FPT *y) {
  for (UIN i = 0; i < n; i++) {
    FPT aux = 0.0;
    for (UIN j = row[i]; j < row[i + 1]; j++) aux = aux + val[j] * x[col[j]];
    y[i] = aux;
  }
}

/* (|A| |x|)_i, the scale of the componentwise parity bound (no reference counterpart). */
ORC_API void orc_abs_csr(UIN n, const UIN *row, const UIN *col, const FPT *val, const FPT *x, FPT *y) {
  for (UIN i = 0; i < n; i++) {
    FPT aux = 0.0;
    for (UIN j = row[i]; j < row[i + 1]; j++) aux += fabs(val[j]) * fabs(x[col[j]]);
    y[i] = aux;
  }
}

/* ---- M:404-425: getErrors ---- */
ORC_API void orc_get_errors(UIN len, const FPT *ar, const FPT *ac, double *aErr, double *rErr, UIN *pos) {
  double maxDif = 0.0, maxVal = 0.0;
  UIN p = 0;
  for (UIN i = 0; i < len; i++) {
    double v = fabs(ar[i]);
    if (v > maxVal) maxVal = v;
    double d = fabs(fabs(ac[i]) - v);
    if (d > maxDif) {
      maxDif = d;
      p = i;
    }
  }
  *aErr = maxDif;
  *rErr = maxDif / maxVal;
  *pos = p;
}

/* ---- AXC, M:619-628: brick row pointer; returns lenAX ---- */
ORC_API UIN orc_axc_brp(UIN n, const UIN *rl, UIN *brp) {
  brp[0] = 0;
  for (UIN r = 0; r < n; r++) {
    UIN bricks = (rl[r] + HBW - 1) / HBW;
    brp[r + 1] = brp[r] + 2 * bricks * HBW;
  }
  return brp[n];
}

/* ---- AXC, M:632-658: element k of row r at brp[r] + 16*(k/8) + k%8, its x copy 8 further.
 * `ax` must arrive zeroed (padding convention). ---- */
ORC_API void orc_axc_ax(UIN n, const UIN *row, const UIN *col, const FPT *val, const FPT *x,
                        const UIN *brp, FPT *ax) {
  for (UIN r = 0; r < n; r++) {
    UIN p = brp[r], c = 0;
    for (UIN j = row[r]; j < row[r + 1]; j++) {
      ax[p] = val[j];
      ax[p + HBW] = x[col[j]];
      if (c == HBW - 1) {
        p += 1 + HBW;
        c = 0;
      } else {
        p++;
        c++;
      }
    }
  }
}

/* ---- AXC kernel, M:711-732 ---- */
ORC_API void orc_axc_spmv(UIN n, const FPT *ax, const UIN *brp, FPT *y) {
  for (UIN r = 0; r < n; r++) {
    FPT sum = 0.0, pro[HBW];
    for (UIN p = brp[r]; p < brp[r + 1]; p += 2 * HBW) {
      for (UIN k = 0; k < HBW; k++) pro[k] = ax[p + k] * ax[p + HBW + k];
      sum = sum + orc_reduce8(pro);
    }
    y[r] = sum;
  }
}

/* ---- K1, M:775-796: rows by length descending.  The reference sorts
 * (ind,val) pairs with glibc qsort and comparator e2.val - e1.val; glibc's
 * qsort is a stable merge sort for arrays of this size, so equal lengths
 * keep ascending row order.  Restated as a stable merge sort. ---- */
typedef struct { UIN ind, val; } orc_pair;
static int orc_cmp(const orc_pair *e1, const orc_pair *e2) { return (int)(e2->val - e1->val); }
static void orc_msort(orc_pair *a, orc_pair *tmp, size_t n) {
  if (n < 2) return;
  size_t h = n / 2;
  orc_msort(a, tmp, h);
  orc_msort(a + h, tmp, n - h);
  size_t i = 0, j = h, k = 0;
  while (i < h && j < n) tmp[k++] = (orc_cmp(&a[i], &a[j]) <= 0) ? a[i++] : a[j++];
  while (i < h) tmp[k++] = a[i++];
  while (j < n) tmp[k++] = a[j++];
  memcpy(a, tmp, n * sizeof(orc_pair));
}
/* permi has (chunkNum+1)*8 entries, zero beyond n (M:851-852). */
ORC_API int orc_k1_permi(UIN n, const UIN *rl, UIN *permi) {
  orc_pair *l = (orc_pair *)malloc((size_t)n * sizeof(orc_pair) + 1);
  orc_pair *t = (orc_pair *)malloc((size_t)n * sizeof(orc_pair) + 1);
  if (!l || !t) {
    free(l);
    free(t);
    return 1;
  }
  for (UIN i = 0; i < n; i++) {
    l[i].ind = i;
    l[i].val = rl[i];
  }
  orc_msort(l, t, n);
  for (UIN i = 0; i < n; i++) permi[i] = l[i].ind;
  free(l);
  free(t);
  return 0;
}

/* ---- K1, M:800-813: nmc = length of each chunk's first (longest) row; chp
 * = running offsets; returns lenVC ---- */
ORC_API UIN orc_k1_nmc_chp(UIN n, const UIN *rl, const UIN *permi, UIN *nmc, UIN *chp) {
  UIN chunkNum = (n + CHK - 1) / CHK, l = 0;
  for (UIN c = 0; c < chunkNum; c++) {
    nmc[c] = rl[permi[c * CHK]];
    l += CHK * nmc[c];
  }
  if (chunkNum) chp[0] = 0;
  for (UIN c = 1; c < chunkNum; c++) chp[c] = chp[c - 1] + nmc[c - 1] * CHK;
  return l;
}

/* ---- K1, M:817-837: column-major inside a chunk; padding stays zero ---- */
ORC_API void orc_k1_valcol(UIN n, const UIN *row, const UIN *col, const FPT *val, const UIN *permi,
                           const UIN *chp, FPT *kval, UIN *kcol) {
  UIN chunkNum = (n + CHK - 1) / CHK;
  for (UIN c = 0; c < chunkNum; c++)
    for (UIN rid = 0; rid < CHK; rid++) {
      UIN r = c * CHK + rid;
      if (r == n) return;
      r = permi[r];
      UIN k = 0;
      for (UIN j = row[r]; j < row[r + 1]; j++, k++) {
        UIN p = chp[c] + k * CHK + rid;
        kval[p] = val[j];
        kcol[p] = col[j];
      }
    }
}

/* ---- K1 kernel, M:943-965 (res in chunk order) ---- */
ORC_API void orc_k1_spmv(UIN chunkNum, const FPT *kval, const UIN *kcol, const UIN *chp, const UIN *nmc,
                         const FPT *x, FPT *res) {
  for (UIN c = 0; c < chunkNum; c++) {
    FPT s[CHK] = {0};
    UIN off = chp[c];
    for (UIN k = 0; k < nmc[c]; k++, off += CHK)
      for (UIN l = 0; l < CHK; l++) s[l] = fma(kval[off + l], x[kcol[off + l]], s[l]);
    for (UIN l = 0; l < CHK; l++) res[c * CHK + l] = s[l];
  }
}

/* ---- M:969-976: orderArrayK1 ---- */
ORC_API void orc_k1_order(UIN n, const UIN *permi, const FPT *dis, FPT *ord) {
  for (UIN i = 0; i < n; i++) ord[permi[i]] = dis[i];
}

/* ---- K1 with integrated reordering, M:1026-1066, mask M:1077-1086 ---- */
ORC_API void orc_k1p_spmv(UIN n, UIN chunkNum, const FPT *kval, const UIN *kcol, const UIN *chp,
                          const UIN *nmc, const UIN *permi, const FPT *x, FPT *y) {
  UIN posDif = chunkNum * CHK - n;
  for (UIN c = 0; c < chunkNum; c++) {
    FPT s[CHK] = {0};
    UIN off = chp[c];
    for (UIN k = 0; k < nmc[c]; k++, off += CHK)
      for (UIN l = 0; l < CHK; l++) s[l] = fma(kval[off + l], x[kcol[off + l]], s[l]);
    UIN lanes = (c + 1 == chunkNum) ? CHK - posDif : CHK;
    for (UIN l = 0; l < lanes; l++) y[permi[c * CHK + l]] = s[l];
  }
}

/* ---- AXT lengths, M:1118-1148.  con[r] = tile*2*ths + subrow*2*thw + column
 * of the row's first slot; slots are counted with rows padded to grpLen
 * (NOC) or packed (COM).  out[0..2] = tileN, lenAX, lenSEC. ---- */
ORC_API void orc_axt_len(UIN n, const UIN *rl, UIN thw, UIN th, int noc, UIN *con, UIN *out) {
  const UIN ths = thw * th, grp = (th == 1) ? thw : th;
  UIN s = 0, cols = 0;
  for (UIN r = 0; r < n; r++) {
    UIN T = ((s + ths) / ths) - 1;
    UIN R = s % th;
    UIN C = ((s + th) / th) - 1 - T * thw;
    con[r] = T * (2 * ths) + R * (2 * thw) + C;
    UIN pos = noc ? ((rl[r] + grp - 1) / grp) * grp : rl[r];
    cols += (pos + th - 1) / th;
    s += pos;
  }
  UIN tiles = (cols + thw - 1) / thw;
  out[0] = tiles;
  out[1] = tiles * 2 * ths;
  if (noc && th == 1) out[2] = tiles;
  else if (noc) out[2] = tiles * thw;
  else out[2] = tiles * ths;
}

/* ---- AXT NOC tileH=1 fill, M:1152-1184 (ax, sec arrive zeroed) ---- */
ORC_API void orc_axt_fill_noc_h1(UIN n, const UIN *row, const UIN *col, const FPT *val, const FPT *x,
                                 UIN thw, const UIN *con, FPT *ax, UIN *sec) {
  for (UIN r = 0; r < n; r++) {
    if (row[r + 1] == row[r]) continue;
    UIN p = con[r], t = p / (2 * thw), c = 0;
    for (UIN j = row[r]; j < row[r + 1]; j++) {
      ax[p] = val[j];
      ax[p + thw] = x[col[j]];
      sec[t] = r;
      p++;
      c++;
      if (c % thw == 0) {
        p += thw;
        t++;
      }
    }
  }
}

/* ---- AXT NOC tileH>1 fill, M:1188-1221: a row fills tile columns top to
 * bottom, th elements per column, then the next column / tile ---- */
ORC_API void orc_axt_fill_noc(UIN n, const UIN *row, const UIN *col, const FPT *val, const FPT *x,
                              UIN thw, UIN th, const UIN *con, FPT *ax, UIN *sec) {
  const UIN ths = thw * th;
  for (UIN r = 0; r < n; r++) {
    if (row[r + 1] == row[r]) continue;
    UIN p = con[r], q = (p / (2 * ths)) * thw + p % thw, c = 0;
    for (UIN j = row[r]; j < row[r + 1]; j++) {
      ax[p] = val[j];
      ax[p + thw] = x[col[j]];
      sec[q] = r;
      p += 2 * thw;
      c++;
      if (c % th == 0) {
        p = p + 1 - 2 * th * thw;
        q++;
        if (p % thw == 0) p += (2 * th - 1) * thw;
      }
    }
  }
}

/* ---- AXT COM tileH=1 fill, M:1225-1260: slot = CSR index; a descriptor
 * (row << log2 bs) | min(remaining-1, bs-1-offset) at each row start and
 * each block start ---- */
ORC_API void orc_axt_fill_com(UIN n, const UIN *row, const UIN *col, const FPT *val, const FPT *x,
                              UIN thw, UIN bs, UIN lg, FPT *ax, UIN *sec) {
  for (UIN r = 0; r < n; r++) {
    UIN len = row[r + 1] - row[r], k = 0;
    for (UIN p = row[r]; p < row[r + 1]; p++, k++) {
      UIN bco = p % bs, tid = p / thw, tco = p % thw;
      ax[tid * 2 * thw + tco] = val[p];
      ax[tid * 2 * thw + tco + thw] = x[col[p]];
      if (k == 0 || bco == 0) {
        UIN q1 = len - k - 1, q2 = bs - 1 - bco;
        sec[tid * thw + tco] = (r << lg) | (q1 > q2 ? q2 : q1);
      }
    }
  }
}

/* ---- AXT NOC tileH=1 kernel, M:1385-1404 (y accumulates) ---- */
ORC_API void orc_axt_noc_h1_spmv(UIN tileN, const FPT *ax, const UIN *sec, FPT *y) {
  FPT pro[HBW];
  for (UIN t = 0; t < tileN; t++) {
    for (UIN k = 0; k < HBW; k++) pro[k] = ax[t * 2 * HBW + k] * ax[t * 2 * HBW + HBW + k];
    y[sec[t]] += orc_reduce8(pro);
  }
}

/* ---- AXT NOC tileH>1 kernel, M:1443-1474: lane sums down th sub-rows,
 * then one accumulation per lane (y accumulates) ---- */
ORC_API void orc_axt_noc_spmv(UIN tileN, UIN th, const FPT *ax, const UIN *sec, FPT *y) {
  for (UIN t = 0; t < tileN; t++) {
    FPT s[HBW] = {0};
    for (UIN k = 0; k < th; k++) {
      const FPT *p = ax + (size_t)t * th * 2 * HBW + (size_t)k * 2 * HBW;
      for (UIN l = 0; l < HBW; l++) s[l] = s[l] + p[l] * p[HBW + l];
    }
    for (UIN l = 0; l < HBW; l++) y[sec[t * HBW + l]] += s[l];
  }
}

/* ---- AXT COM tileH=1 kernel as the reference computes it, M:1517-1566,
 * including its defects: descriptors equal to 0 are skipped (row 0 with an
 * offset of 0, README.md:33) and a segment sum is a difference of block
 * prefix sums.  The per-tile prefix scan is the reference's three masked
 * permute-adds (shifts 1, 2, 4), then the carry of the previous tile.
 * Kept to reproduce the reference's output, defects included. ---- */
ORC_API int orc_axt_com_h1_ref(UIN bs, UIN lg, UIN tileN, UIN lenSEC, const FPT *ax, const UIN *sec,
                               FPT *y) {
  const UIN bn = (tileN * HBW + bs - 1) / bs, tpb = bs / HBW;
  const size_t lenAX = (size_t)tileN * 2 * HBW;
  FPT *b1 = (FPT *)calloc((size_t)bn * bs + 1, sizeof(FPT));
  FPT *b2 = (FPT *)calloc((size_t)bn * bs + 1, sizeof(FPT));
  if (!b1 || !b2) {
    free(b1);
    free(b2);
    return 1;
  }
  for (UIN b = 0; b < bn; b++) {
    FPT acu = 0.0;
    for (UIN t = 0; t < tpb; t++) {
      size_t pa = (size_t)b * tpb * 2 * HBW + (size_t)t * 2 * HBW;
      size_t pb = (size_t)b * bs + (size_t)t * HBW;
      FPT v[HBW], w[HBW];
      for (UIN l = 0; l < HBW; l++) v[l] = (pa + HBW + l < lenAX) ? ax[pa + l] * ax[pa + HBW + l] : 0.0;
      for (UIN l = 0; l < HBW; l++) b1[pb + l] = v[l];
      for (UIN l = 0; l < HBW; l++) w[l] = (l >= 1) ? v[l] + v[l - 1] : v[l];
      for (UIN l = 0; l < HBW; l++) v[l] = w[l];
      for (UIN l = 0; l < HBW; l++) w[l] = (l >= 2) ? v[l] + v[l - 2] : v[l];
      for (UIN l = 0; l < HBW; l++) v[l] = w[l];
      for (UIN l = 0; l < HBW; l++) w[l] = (l >= 4) ? v[l] + v[l - 4] : v[l];
      for (UIN l = 0; l < HBW; l++) b2[pb + l] = w[l] + acu;
      acu = b2[pb + HBW - 1];
    }
    UIN sp = b * bs, ep = (b + 1) * bs;
    ep = ep > lenSEC ? lenSEC : ep;
    for (UIN p = sp; p < ep; p++) {
      UIN ro = sec[p];
      if (ro != 0) {
        UIN r = ro >> lg, o = ro & (bs - 1);
        y[r] += b2[p + o] - b2[p] + b1[p];
      }
    }
  }
  free(b1);
  free(b2);
  return 0;
}
