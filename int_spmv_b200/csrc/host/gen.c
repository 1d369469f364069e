/*
 * gen.c - seeded generator of the banded FEM-like matrices of the batched
 * benchmark workload (no reference counterpart: the reference reads its
 * matrices from files, and the ones its job scripts name are not available).
 *
 * Row r of an n x n matrix holds rl[r] entries, rl uniform in [rl_lo, rl_hi]
 * (at most n): the diagonal plus rl-1 distinct columns drawn uniformly from
 * [r - band*rl, r + band*rl] clipped to [0, n) without r.  Off-diagonal values
 * are N(0,1); the diagonal is |sum of the row's off-diagonals| + 1.  Columns
 * are ascending within each row.
 *
 * Random numbers: SplitMix64 (Steele, Lea and Flood, "Fast splittable
 * pseudorandom number generators", OOPSLA 2014), one independent stream per
 * row keyed by (seed, row), so the result does not depend on the thread
 * count.  The distinct columns are a uniform k-subset by Floyd's algorithm
 * (Bentley and Floyd, "Programming pearls: a sample of brilliance", CACM
 * 1987) over a per-thread bitmap; normals by the Box-Muller transform.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "intspmv.h"

#define API __attribute__((visibility("default")))

typedef struct { uint64_t s; } gen_rng;

static inline uint64_t gen_next(gen_rng *g) {
  uint64_t z = (g->s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static inline gen_rng gen_stream(uint64_t seed, uint64_t row, uint64_t salt) {
  gen_rng g = {seed * 0xD1342543DE82EF95ull + salt};
  g.s ^= gen_next(&g) + row * 0xA24BAED4963EE407ull;
  (void)gen_next(&g);
  return g;
}
/* uniform integer in [0, m), m > 0 (64-bit draw, bias below 2^-32) */
static inline uint32_t gen_below(gen_rng *g, uint32_t m) {
  return (uint32_t)(((gen_next(g) >> 32) * (uint64_t)m) >> 32);
}
/* uniform in (0, 1] */
static inline double gen_unit(gen_rng *g) { return ((double)(gen_next(g) >> 11) + 1.0) * 0x1.0p-53; }
static inline double gen_normal(gen_rng *g) {
  const double u1 = gen_unit(g), u2 = gen_unit(g);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586476925 * u2);
}

API int ispmv_gen_banded(UIN n, uint64_t seed, UIN rl_lo, UIN rl_hi, UIN band, str_matCSR *out) {
  if (!out || n == 0 || rl_lo == 0 || rl_hi < rl_lo || band == 0) return ISPMV_ERR_ARG;
  memset(out, 0, sizeof *out);
  UIN *rl = (UIN *)malloc(((size_t)n + 1) * sizeof(UIN));
  UIN *row = (UIN *)malloc(((size_t)n + 1) * sizeof(UIN));
  if (!rl || !row) { free(rl); free(row); return ISPMV_ERR_OOM; }
  long long r;
#pragma omp parallel for schedule(static)
  for (r = 0; r < (long long)n; r++) {
    gen_rng g = gen_stream(seed, (uint64_t)r, 1);
    UIN l = rl_lo + gen_below(&g, rl_hi - rl_lo + 1);
    rl[r] = l < n ? l : n;
  }
  uint64_t nnz = 0;
  for (UIN i = 0; i < n; i++) {
    row[i] = (UIN)nnz;
    nnz += rl[i];
    if (nnz > 0xFFFFFFFFull) { free(rl); free(row); return ISPMV_ERR_OVERFLOW; }
  }
  row[n] = (UIN)nnz;
  UIN *col = (UIN *)malloc((size_t)(nnz ? nnz : 1) * sizeof(UIN));
  FPT *val = (FPT *)malloc((size_t)(nnz ? nnz : 1) * sizeof(FPT));
  if (!col || !val) { free(rl); free(row); free(col); free(val); return ISPMV_ERR_OOM; }
  const uint64_t wmax = (uint64_t)2 * band * rl_hi + 1;  /* widest window */
  const size_t words = (size_t)((wmax < n ? wmax : n) / 64 + 1);
  int oom = 0;
#pragma omp parallel
  {
    uint64_t *bits = (uint64_t *)calloc(words, sizeof(uint64_t));
    if (!bits) {
#pragma omp atomic write
      oom = 1;
    }
#pragma omp for schedule(dynamic, 4096)
    for (r = 0; r < (long long)n; r++) {
      if (!bits) continue;
      gen_rng g = gen_stream(seed, (uint64_t)r, 2);
      const UIN l = rl[r];
      const long long w = (long long)band * l;
      const long long lo = r - w < 0 ? 0 : r - w;
      const long long hi = r + w > (long long)n - 1 ? (long long)n - 1 : r + w;
      const uint32_t m = (uint32_t)(hi - lo);  /* candidates: the window without r */
      const uint32_t k = l - 1;                /* k <= m: the window holds at least l columns */
      for (uint32_t j = m - k; j < m; j++) {   /* Floyd: a uniform k-subset of [0, m) */
        const uint32_t t = gen_below(&g, j + 1);
        if (bits[t >> 6] >> (t & 63) & 1u) bits[j >> 6] |= 1ull << (j & 63);
        else bits[t >> 6] |= 1ull << (t & 63);
      }
      UIN *c = col + row[r];
      FPT *v = val + row[r];
      UIN q = 0, dpos = 0;
      int placed = 0;  /* the diagonal's slot has been reserved */
      double sum = 0.0;
      for (size_t wd = 0; wd <= (size_t)(m ? (m - 1) >> 6 : 0) && wd < words; wd++) {
        uint64_t b = bits[wd];
        bits[wd] = 0;
        while (b) {
          const uint32_t i = (uint32_t)(wd * 64 + (uint64_t)__builtin_ctzll(b));
          b &= b - 1;
          const long long cc = lo + i + (lo + i >= r ? 1 : 0);  /* skip the diagonal */
          if (!placed && cc > r) {                              /* the diagonal's place */
            dpos = q++;
            placed = 1;
          }
          c[q] = (UIN)cc;
          const double x = gen_normal(&g);
          v[q++] = x;
          sum += x;
        }
      }
      if (!placed) dpos = q++;  /* every column below r: the diagonal comes last */
      c[dpos] = (UIN)r;
      v[dpos] = fabs(sum) + 1.0;
    }
    free(bits);
  }
  if (oom) { free(rl); free(row); free(col); free(val); return ISPMV_ERR_OOM; }
  out->nrows = n;
  out->nnz = (UIN)nnz;
  out->row = row;
  out->col = col;
  out->val = val;
  out->rl = rl;
  return ispmv_csr_stats(out);
}
