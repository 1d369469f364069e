/*
 * ref_shim.h - TEST INFRASTRUCTURE ONLY.  Force-included (gcc -include) when
 * the reference intSpmv_main.c is compiled where it lies, so that GCC builds
 * it.  The reference targets ICC (ic.sh:42-43); this shim supplies what GCC
 * lacks without touching the reference source:
 *   1. ICC-only "lo" gather/scatter intrinsics (intSpmv_main.c:957,1040,1046,
 *      1057,1063) mapped to the 256-bit-index forms on the low 8 indices.
 *   2. Aligned 512-bit load/store intrinsics mapped to unaligned ones: the
 *      reference issues them at 32-byte offsets and on an unaligned stack
 *      array (intSpmv_main.c:956,1039,1045,1464); ICC emits unaligned moves.
 *   3. _mm_malloc routed to ref_shim_malloc: 64-byte aligned, with 16 KiB of
 *      zeroed slack after every block (absorbs the 32-byte over-read at
 *      intSpmv_main.c:956 and the compacted kernel's read past lenAX at
 *      intSpmv_main.c:1538), zero-filled while `ref_shim_zero` is set (the
 *      reference relies on fresh pages being zero for AXC/K1 padding,
 *      intSpmv_main.c:684,877-878), and optionally tracked so a harness can
 *      free the per-call scratch the compacted kernel never frees
 *      (intSpmv_main.c:1529-1530).
 * MKL is not installed; shim/mkl.h declares stubs that abort if called.
 */
#ifndef REF_SHIM_H
#define REF_SHIM_H
#include <immintrin.h>
#include <stdlib.h>
#include <string.h>

#define _mm512_i32logather_pd(idx, base, scale) \
  _mm512_i32gather_pd(_mm512_castsi512_si256(idx), (base), (scale))
#define _mm512_i32loscatter_pd(base, idx, v, scale) \
  _mm512_i32scatter_pd((base), _mm512_castsi512_si256(idx), (v), (scale))
#define _mm512_mask_i32loscatter_pd(base, mask, idx, v, scale) \
  _mm512_mask_i32scatter_pd((base), (mask), _mm512_castsi512_si256(idx), (v), (scale))

#define _mm512_load_pd(p) _mm512_loadu_pd((const void *)(p))
#define _mm512_store_pd(p, v) _mm512_storeu_pd((void *)(p), (v))
#define _mm512_load_epi32(p) _mm512_loadu_si512((const void *)(p))
#define _mm512_store_epi32(p, v) _mm512_storeu_si512((void *)(p), (v))

#define REF_SHIM_SLACK 16384u
#define REF_SHIM_MAX_TRACK 256
extern int ref_shim_zero;
extern int ref_shim_tracking;
extern int ref_shim_ntrack;
extern void *ref_shim_track[REF_SHIM_MAX_TRACK];

static inline void *ref_shim_malloc(size_t sz, size_t al) {
  void *p = NULL;
  if (al < sizeof(void *)) al = sizeof(void *);
  if (posix_memalign(&p, al, sz + REF_SHIM_SLACK) != 0) return NULL;
  if (ref_shim_zero) memset(p, 0, sz + REF_SHIM_SLACK);
  else memset((char *)p + sz, 0, REF_SHIM_SLACK);
  if (ref_shim_tracking && ref_shim_ntrack < REF_SHIM_MAX_TRACK) ref_shim_track[ref_shim_ntrack++] = p;
  return p;
}
#undef _mm_malloc
#undef _mm_free
#define _mm_malloc(sz, al) ref_shim_malloc((size_t)(sz), (size_t)(al))
#define _mm_free(p) free(p)

#endif
