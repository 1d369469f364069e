/*
 * intspmv.h - C ABI of int_spmv_b200, a B200 (sm_100a) SpMV library that is a
 * drop-in for the C entry points and sparse formats of edoardoCB/int_spmv.
 *
 * Every reference citation below is `intSpmv_main.c:<line>` of that project
 * (abbreviated `M:<line>`).  The reference is one C translation unit whose
 * functions are all `static`; its "C entry points" are the signatures and
 * struct layouts reproduced here, made non-static and `extern "C"`.
 *
 * Three layers:
 *   1. Host format builders with the reference's signatures and allocation
 *      contract (arrays malloc'd inside the struct, caller frees with free()).
 *      Pointer, index and reorder arrays are bit-exact to the reference.
 *      Status-returning `ispmv_build_*` forms sit beside the compat forms,
 *      which, like the reference, print and exit(EXIT_FAILURE) on error.
 *   2. Kernels with the reference's names and signatures on HOST pointers
 *      (`cf_CSR`, `int_axc`, ...): each call copies its inputs to the GPU,
 *      runs the sm_100a kernel and copies the result back.  `ompNT` is
 *      accepted and ignored.  The same kernels on DEVICE pointers are the
 *      `ispmv_dev_*` functions (stream-ordered, status-returning).
 *   3. Plans (`ispmv_plan_*`): a format uploaded once to HBM as value and
 *      column-index streams, then y = A*x (+ beta*y) for a fresh x on every
 *      call, in FP64 or a reduced-byte form (FP32 values, FP64 accumulation).
 *
 * All functions returning `int` return an ISPMV_* status; 0 is success.
 */
#ifndef INTSPMV_H
#define INTSPMV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------------
 * Compile-time configuration of the reference (M:51-109, ic.sh:43).  FPT is
 * the value type, chosen as the reference chooses it: FP_TYPE=FP_DOUBLE (the
 * default) or FP_TYPE=FP_FLOAT on the compile line (or ISPMV_FPT_FLOAT).
 * The reference's own FP32 build does not compile (the M:207 typo, `_pd`
 * intrinsics); here it does.  With FPT = float the structs hold float
 * values and the layer-1 and layer-2 names below resolve to their `_f32`
 * symbols (the same library exports both): values, x and y are FP32, every
 * product and sum is computed in FP64 and y is rounded to FP32 once.  The
 * device plans (layer 3) and the GPU format builders are FP64 only.
 * ------------------------------------------------------------------------ */
#ifndef FP_FLOAT
#define FP_FLOAT 1  /* M:51-53 */
#endif
#ifndef FP_DOUBLE
#define FP_DOUBLE 2 /* M:57-59 */
#endif
#if defined(FP_TYPE) && !defined(ISPMV_FPT_FLOAT)
#if FP_TYPE == FP_FLOAT
#define ISPMV_FPT_FLOAT 1
#endif
#endif
#ifdef ISPMV_FPT_FLOAT
typedef float FPT;         /* M:63-66 */
#else
typedef double FPT;        /* M:70-73 */
#endif
typedef unsigned int UIN;  /* M:77-79 */
#define ISPMV_HBRICK_SIZE 8u /* M:101-103: brick / tile width */
#define ISPMV_CHUNK_SIZE 8u  /* M:107-109: K1 chunk height */

/* Status codes (the reference exits instead: M:171-179). */
#define ISPMV_OK 0
#define ISPMV_ERR_ARG 1         /* bad argument or malformed matrix */
#define ISPMV_ERR_OOM 2         /* host or device allocation failed */
#define ISPMV_ERR_CUDA 3        /* a CUDA runtime call failed */
#define ISPMV_ERR_TIMEOUT 4     /* a bounded device wait gave up */
#define ISPMV_ERR_UNSUPPORTED 5 /* valid for the reference, not implemented */
#define ISPMV_ERR_OVERFLOW 6    /* a u32 length or index would overflow */

#ifdef ISPMV_FPT_FLOAT
/* FPT = float: every function whose arguments hold FPT resolves to its FP32
 * symbol. */
#define ispmv_csr_stats ispmv_csr_stats_f32
#define printMatrixStats printMatrixStats_f32
#define ispmv_matrix_read ispmv_matrix_read_f32
#define matrixReading matrixReading_f32
#define ispmv_matrix_write ispmv_matrix_write_f32
#define ispmv_csr_free ispmv_csr_free_f32
#define ispmv_build_csr ispmv_build_csr_f32
#define getFormatDataCSR getFormatDataCSR_f32
#define ispmv_build_axc ispmv_build_axc_f32
#define getFormatDataAXC getFormatDataAXC_f32
#define ispmv_build_k1 ispmv_build_k1_f32
#define getFormatDataK1 getFormatDataK1_f32
#define ispmv_build_axt ispmv_build_axt_f32
#define getFormatDataAXT getFormatDataAXT_f32
#define ispmv_build_axc_cols ispmv_build_axc_cols_f32
#define ispmv_build_axt_cols ispmv_build_axt_cols_f32
#define ispmv_free_axc ispmv_free_axc_f32
#define ispmv_free_k1 ispmv_free_k1_f32
#define ispmv_free_axt ispmv_free_axt_f32
#define getErrors getErrors_f32
#define initVec initVec_f32
#define fill_array fill_array_f32
#define ispmv_dev_cf_csr ispmv_dev_cf_csr_f32
#define ispmv_dev_int_axc ispmv_dev_int_axc_f32
#define ispmv_dev_int_k1 ispmv_dev_int_k1_f32
#define ispmv_dev_order_k1 ispmv_dev_order_k1_f32
#define ispmv_dev_int_k1p ispmv_dev_int_k1p_f32
#define ispmv_dev_int_axt_noc_h1 ispmv_dev_int_axt_noc_h1_f32
#define ispmv_dev_int_axt_noc ispmv_dev_int_axt_noc_f32
#define ispmv_dev_int_axt_com_h1 ispmv_dev_int_axt_com_h1_f32
#define cf_CSR cf_CSR_f32
#define int_axc int_axc_f32
#define int_k1 int_k1_f32
#define orderArrayK1 orderArrayK1_f32
#define int_k1p int_k1p_f32
#define int_axt_noc_h1 int_axt_noc_h1_f32
#define int_axt_noc int_axt_noc_f32
#define int_axt_com_h1 int_axt_com_h1_f32
#define test_cf_CSR test_cf_CSR_f32
#define test_int_AXC test_int_AXC_f32
#define test_int_k1 test_int_k1_f32
#define test_int_k1p test_int_k1p_f32
#define test_int_axt_noc_h1 test_int_axt_noc_h1_f32
#define test_int_axt_noc test_int_axt_noc_f32
#define test_int_axt_com_h1 test_int_axt_com_h1_f32
#endif

/* ---------------------------------------------------------------------------
 * Reference structs, field for field (same order, same types).
 * ------------------------------------------------------------------------ */
/* M:183 - input CSR plus row statistics; `rl` is filled by the stats pass
 * (M:253-262).  rowStart/rowEnd are only used by the MKL rows (M:324-357). */
typedef struct {
  UIN nrows; UIN nnz; UIN rmin; FPT rave; UIN rmax; FPT rsd; UIN bw;
  FPT *val; UIN *row; UIN *rowStart; UIN *rowEnd; UIN *col; UIN *rl;
} str_matCSR;

/* M:306 - per-format name, memory footprint [B], occupancy, conversion time */
typedef struct { char name[24]; double mfp; double beta; double ct; } str_formatData;

/* M:400 - error of a result against the CSR oracle (M:404-425) */
typedef struct { double aErr; double rErr; UIN pos; } str_err;

/* M:429 - one row of the kernels' results table */
typedef struct { char name[25]; double et; double ot; double flops; str_err sErr; } str_res;

/* M:615 - AXC: rows of 8-wide bricks, each 8 values then 8 x copies */
typedef struct { UIN nrows; UIN nnz; UIN lenAX; UIN lenBRP; FPT *ax; UIN *brp; } str_matAXC;

/* M:771 - K1: rows sorted by length, 8-row chunks stored column-major */
typedef struct {
  UIN nrows; UIN nnz; UIN chunkNum; UIN lenVC;
  UIN *permi; UIN *nmc; UIN *chp; FPT *val; UIN *col;
} str_matK1;

/* M:1114 - AXT: tiles of tileH sub-rows x (8 values + 8 x copies) */
typedef struct {
  UIN nrows; UIN nnz; char mode[8]; UIN tileHW; UIN tileH; UIN logTH; UIN tileN;
  UIN lenAX; UIN lenSEC; UIN lenCON; UIN log; FPT *ax; UIN *sec; UIN *con;
} str_matAXT;

/* ---------------------------------------------------------------------------
 * Layer 1: host format builders.
 * ------------------------------------------------------------------------ */

/* Fills rl[i] = row[i+1]-row[i] and rmin/rave/rmax/rsd/bw of `csr`
 * (the computation of printMatrixStats, M:253-278, without its .sta file).
 * Also validates the CSR (row pointers monotone, row[n]==nnz, col<nrows). */
int ispmv_csr_stats(str_matCSR *csr);

/* printMatrixStats, M:253-302: ispmv_csr_stats plus the `<name>.sta` file,
 * written beside the matrix file (the extension after the last '.' of the
 * file name is replaced; the reference's strtok rule breaks on dotted paths,
 * M:280-287). */
void printMatrixStats(const char *matFileName, str_matCSR *matCSR);

/* matrixReading, M:187-249: reads a `.csr` text file ("n nnz", nnz lines
 * "val col", n+1 row pointers) or a `.bin` file (u32 n, u32 nnz, FPT
 * val[nnz], u32 col[nnz], u32 row[n+1]).  Arrays are malloc'd, rl included
 * (unfilled until the stats pass).  ispmv_matrix_read returns a status;
 * matrixReading exits on error like the reference. */
int ispmv_matrix_read(const char *matFileName, str_matCSR *out);
str_matCSR matrixReading(const char *matFileName);
/* Writes `csr` as a .csr (text) or .bin file, chosen by the extension. */
int ispmv_matrix_write(const char *matFileName, const str_matCSR *csr);
/* Frees every array of a CSR produced by ispmv_matrix_read. */
void ispmv_csr_free(str_matCSR *csr);

/* getFormatDataCSR, M:324-357: rowStart/rowEnd copies and the CSR row of
 * the formats table (memory footprint includes the x vector, M:350). */
int ispmv_build_csr(str_matCSR *csr, str_formatData *fd);
str_formatData getFormatDataCSR(str_matCSR *matCSR);

/* getFormatDataAXC, M:662-707.  brp (M:619-628) is calloc'd, ax (M:632-658)
 * is 64-byte aligned with its padding zeroed.  Requires csr.rl. */
int ispmv_build_axc(UIN ompNT, const str_matCSR *csr, const FPT *vec, str_matAXC *out,
                    str_formatData *fd);
str_formatData getFormatDataAXC(const UIN ompNumThreads, const str_matCSR matCSR,
                                const FPT *vec, str_matAXC *matAXC);

/* getFormatDataK1, M:841-905.  permi (M:782-796) orders rows by length
 * descending, ties by ascending row id (the order glibc's qsort gives the
 * reference, M:775-778); nmc/chp (M:800-813); val/col (M:817-837) padding
 * zeroed.  `blockSize` is unused, as in the reference. */
int ispmv_build_k1(UIN blockSize, const str_matCSR *csr, const FPT *vec, str_matK1 *out,
                   str_formatData *fd);
str_formatData getFormatDataK1(const UIN blockSize, const str_matCSR matCSR,
                               const FPT *vec, str_matK1 *matK1);

/* getFormatDataAXT, M:1275-1381.  mode "NOC" (uncompacted, any tileH >= 1)
 * or "COM" (compacted, tileH == 1 and bs a power of two in [2, 512]; the
 * reference leaves COM with tileH > 1 unimplemented, M:1338-1362).
 * con (M:1118-1148), ax and sec (M:1152-1260) are bit-exact; ax and sec
 * padding is zero (M:1304-1305). */
int ispmv_build_axt(UIN ompNT, UIN bs, UIN thw, UIN th, const char *mode,
                    const str_matCSR *csr, const FPT *vec, str_matAXT *out,
                    str_formatData *fd);
str_formatData getFormatDataAXT(const UIN ompNT, const UIN bs, const UIN thw, const UIN th,
                                const char *mode, const str_matCSR matCSR, const FPT *vec,
                                str_matAXT *matAXT);

/* Column-index companions (no reference counterpart): the reference bakes
 * x into ax (M:644, M:1171, M:1207, M:1247), so its AXC/AXT kernels never
 * gather x.  The companion holds, for every value slot of ax, the column of
 * that value: axi[s] is the column of ax[(s/thw)*2*thw + s%thw];
 * length lenAX/2; padding slots hold column 0 (their value is 0.0).
 * *axi is malloc'd; the caller frees it. */
int ispmv_build_axc_cols(UIN ompNT, const str_matCSR *csr, const str_matAXC *axc, UIN **axi);
int ispmv_build_axt_cols(UIN ompNT, const str_matCSR *csr, const str_matAXT *axt, UIN **axi);

#ifndef ISPMV_FPT_FLOAT
/* Block-diagonal CSR of `count` square matrices (no reference counterpart:
 * the batched path).  Matrix m's rows and columns start at off[m]; off has
 * count+1 entries.  Arrays are malloc'd (ispmv_csr_free); rl and the
 * statistics are filled. */
int ispmv_csr_blockdiag(UIN count, const str_matCSR *mats, str_matCSR *out, UIN *off);
/* Seeded banded FEM-like matrix (no reference counterpart; a benchmark
 * workload generator): row r holds rl uniform in [rl_lo, rl_hi] (at most n)
 * entries, the diagonal plus rl-1 distinct columns uniform in
 * [r - band*rl, r + band*rl] clipped to [0, n); off-diagonals N(0,1), the
 * diagonal |off-diagonal sum| + 1; ascending columns.  Arrays malloc'd
 * (ispmv_csr_free); rl and statistics filled.  Deterministic in (n, seed,
 * rl_lo, rl_hi, band) whatever the thread count. */
int ispmv_gen_banded(UIN n, uint64_t seed, UIN rl_lo, UIN rl_hi, UIN band, str_matCSR *out);
#endif

/* Frees the arrays a builder allocated and zeroes the struct. */
void ispmv_free_axc(str_matAXC *m);
void ispmv_free_k1(str_matK1 *m);
void ispmv_free_axt(str_matAXT *m);

/* getErrors, M:404-425: aErr = max_i | |res_i| - |ref_i| |, rErr = aErr /
 * max_i |ref_i|, pos = first argmax. */
void getErrors(const UIN len, const FPT *ar, const FPT *ac, str_err *sErr);
void initVec(const UIN len, FPT *vec); /* M:361-367: vec[i] = i */
/* fill_array, M:371-378: array[i] = val (host memory, ompNT threads). */
void fill_array(const UIN ompNT, const UIN len, FPT val, FPT *array);

/* ---------------------------------------------------------------------------
 * Layer 2a: kernels on DEVICE pointers (stream-ordered; `stream` is a
 * cudaStream_t, NULL for the legacy default stream).  Same arithmetic and
 * accumulation contract as the reference kernel each one replaces; AXT
 * kernels accumulate into y (the caller zeroes it, M:1421,1492,1591).
 * ------------------------------------------------------------------------ */
int ispmv_dev_cf_csr(UIN nrows, const UIN *row, const UIN *col, const FPT *val, const FPT *vec,
                     FPT *res, void *stream);                                   /* M:382 */
int ispmv_dev_int_axc(UIN nrows, const FPT *ax, const UIN *brp, FPT *y, void *stream); /* M:711 */
int ispmv_dev_int_k1(UIN chunkNum, const FPT *val, const UIN *col, const UIN *chp,
                     const UIN *nmc, const FPT *vec, FPT *res, void *stream);   /* M:943 */
int ispmv_dev_order_k1(UIN len, const UIN *permi, const FPT *arrDis, FPT *arrOrd,
                       void *stream);                                           /* M:969 */
/* `mask` is the reference's tail mask for the last chunk (M:1077-1086):
 * bit i set = lane i of the last chunk is a real row. */
int ispmv_dev_int_k1p(unsigned char mask, UIN chunkNum, const FPT *val, const UIN *col,
                      const UIN *chp, const UIN *nmc, const UIN *permi, const FPT *vec,
                      FPT *res, void *stream);                                  /* M:1026 */
int ispmv_dev_int_axt_noc_h1(UIN tileNum, const FPT *ax, const UIN *rwp, FPT *y,
                             void *stream);                                     /* M:1385 */
int ispmv_dev_int_axt_noc(UIN tileNum, UIN tileHeight, const FPT *ax, const UIN *rwp, FPT *y,
                          void *stream);                                        /* M:1443 */
/* Compacted AXT (M:1517).  Computes the true segmented sum of every
 * segment, including row-0 segments whose descriptor encodes as 0 (the
 * reference skips those, M:1555) and without reading past lenAX. */
int ispmv_dev_int_axt_com_h1(UIN bn, UIN bs, UIN log, UIN thw, UIN tn, UIN lenAX, UIN lenRWP,
                             const FPT *ax, const UIN *rwp, FPT *y, void *stream);

/* K1 SpMV in original row order, y[permi[i]] = (chunk-order product)[i],
 * that allocates nothing.  No counterpart in the reference (whose int_k1
 * writes a caller-provided result array that orderArrayK1 then reorders).
 * For callers that cannot call cudaMalloc - a solver loop whose memory is
 * fixed before it starts, or a host that gives the library no allocator -
 * the chunk-order intermediate lives in a static device array of
 * ISPMV_K1_NOALLOC_MAX_ROWS doubles (8 MiB), held by every GPU that loads
 * the library until the process exits.  Arrays are those of str_matK1 on
 * the device; vec and y have nrows entries; chunkNum = ceil(nrows / 8).
 * More rows than the maximum, or a null array, is rejected with
 * ISPMV_ERR_ARG before anything is launched.  The first call in a device's
 * context looks up the array's device address (cudaGetSymbolAddress); the
 * address is kept for that context and looked up again in a new one (after
 * cudaDeviceReset, say), so make the first call on each device, and the
 * first after a reset, before any stream capture.  Calls share the
 * array: calls that overlap on the GPU (concurrent streams, or several host
 * threads) race and must be serialised by the caller.  Nothing needs
 * clearing between calls: every call writes the part of the array it reads. */
#define ISPMV_K1_NOALLOC_MAX_ROWS (1u << 20)
#ifndef ISPMV_FPT_FLOAT
int ispmv_dev_k1_spmv_noalloc(UIN nrows, UIN chunkNum, const FPT *val, const UIN *col, const UIN *chp,
                              const UIN *nmc, const UIN *permi, const FPT *vec, FPT *y, void *stream);
#endif

/* ---------------------------------------------------------------------------
 * Layer 2b: the reference's kernels by name on HOST pointers.  Each call
 * copies its inputs to the current GPU, runs the ispmv_dev_* kernel and
 * copies the result back (synchronous).  Errors print and exit, as the
 * reference does.  `ompNT` is ignored.
 * ------------------------------------------------------------------------ */
void cf_CSR(const str_matCSR matCSR, const FPT *vec, FPT *res);                 /* M:382 */
void int_axc(const UIN ompNT, const UIN nrows, const FPT *ax, const UIN *brp, FPT *y); /* M:711 */
void int_k1(const UIN ompNT, const UIN chunkNum, const FPT *val, const UIN *col,
            const UIN *chp, const UIN *nmc, const FPT *vec, FPT *res);         /* M:943 */
void orderArrayK1(const UIN ompNT, const UIN len, const UIN *permi, const FPT *arrDis,
                  FPT *arrOrd);                                                 /* M:969 */
void int_k1p(const UIN ompNT, const unsigned char mask, const UIN chunkNum, const FPT *val,
             const UIN *col, const UIN *chp, const UIN *nmc, const UIN *permi,
             const FPT *vec, FPT *res);                                         /* M:1026 */
void int_axt_noc_h1(const UIN ompNT, const UIN tileNum, const FPT *ax, const UIN *rwp,
                    FPT *y);                                                    /* M:1385 */
void int_axt_noc(const UIN ompNT, const UIN tileNum, const UIN tileHeight, const FPT *ax,
                 const UIN *rwp, FPT *y);                                       /* M:1443 */
void int_axt_com_h1(const UIN ompNT, const UIN bn, const UIN bs, const UIN log, const UIN thw,
                    const UIN tn, const UIN lenAX, const UIN lenRWP, const FPT *ax,
                    const UIN *rwp, FPT *y);                                    /* M:1517 */

/* ---------------------------------------------------------------------------
 * Layer 2c: the reference's per-kernel harness (test_*, M:433-1609), as a
 * reference caller times and checks kernels.  Each uploads its arrays to
 * the GPU once, runs the kernel NUM_ITE times (AXT kernels on a y zeroed
 * before every run, outside the timed region, as fill_array does, M:1420),
 * and fills str_res: name (the reference's string), et = mean time of one
 * kernel run in seconds (CUDA events around the launch on the GPU),
 * ot = mean time of the reorder pass (test_int_k1 only: orderArrayK1, M:1001)
 * else 0, flops = 2*nnz / et, and sErr = getErrors(nrows, ref, result).
 * The arrays are those the reference-named builders produce.  Errors print
 * and exit like the reference.
 * ------------------------------------------------------------------------ */
#define ISPMV_NUM_ITE_DEFAULT 250u /* M:93-95 */
/* Runs per test_* call: $ISPMV_NUM_ITE when set, else ISPMV_NUM_ITE_DEFAULT;
 * ispmv_set_num_ite(n) overrides both (0 restores them). */
void ispmv_set_num_ite(UIN n);
UIN ispmv_get_num_ite(void);
str_res test_cf_CSR(const str_matCSR matCSR, const FPT *vec, const FPT *ref);            /* M:433 */
str_res test_int_AXC(const UIN ompNT, const str_matAXC matAXC, const FPT *ref);          /* M:736 */
str_res test_int_k1(const UIN ompNT, const str_matK1 matK1, const FPT *vec, const FPT *ref); /* M:980 */
str_res test_int_k1p(const UIN ompNT, const str_matK1 matK1, const FPT *vec, const FPT *ref); /* M:1070 */
str_res test_int_axt_noc_h1(const UIN ompNT, const str_matAXT matAXT, const FPT *ref);   /* M:1408 */
str_res test_int_axt_noc(const UIN ompNT, const str_matAXT matAXT, const FPT *ref);      /* M:1478 */
str_res test_int_axt_com_h1(const UIN ompNT, const UIN bs, const str_matAXT matAXT,
                            const FPT *ref);                                             /* M:1570 */

#ifndef ISPMV_FPT_FLOAT
/* Format conversion on the GPU (no reference counterpart: the reference
 * converts on the host, getFormatDataAXT M:1275-1381).  Builds the same
 * con/ax/sec arrays as getFormatDataAXT, bit for bit, from a CSR matrix and
 * x in DEVICE memory (d_row n+1, d_col/d_val nnz, d_x n).  The struct's
 * con/ax/sec are device pointers, to be released with ispmv_dev_axt_free;
 * fd->ct is the conversion's GPU time in seconds.  Synchronises `stream`.
 * Feed the result to ispmv_dev_int_axt_noc_h1 / _noc / _com_h1. */
int ispmv_dev_build_axt(UIN bs, UIN thw, UIN th, const char *mode, UIN n, UIN nnz, const UIN *d_row,
                        const UIN *d_col, const FPT *d_val, const FPT *d_x, str_matAXT *m,
                        str_formatData *fd, void *stream);
int ispmv_dev_axt_free(str_matAXT *m);
/* Copies a device-built AXT's con/ax/sec (lenCON/lenAX/lenSEC entries) into
 * caller buffers, host or device (NULL skips one); synchronises `stream`. */
int ispmv_dev_axt_export(const str_matAXT *m, UIN *con, FPT *ax, UIN *sec, void *stream);
/* getFormatDataK1 (M:841-905) on the GPU, likewise: permi/nmc/chp/val/col
 * bit for bit the host builder's, from device CSR arrays; device pointers in
 * the struct (ispmv_dev_k1_free); feed them to ispmv_dev_int_k1 / _k1p. */
int ispmv_dev_build_k1(UIN n, UIN nnz, const UIN *d_row, const UIN *d_col, const FPT *d_val, str_matK1 *m,
                       str_formatData *fd, void *stream);
int ispmv_dev_k1_free(str_matK1 *m);
/* Copies permi ((chunkNum+1)*8), nmc, chp (chunkNum) and val, col (lenVC)
 * into caller buffers (NULL skips one); synchronises `stream`. */
int ispmv_dev_k1_export(const str_matK1 *m, UIN *permi, UIN *nmc, UIN *chp, FPT *val, UIN *col, void *stream);

/* ---------------------------------------------------------------------------
 * Layer 3: plans - a format resident in HBM as value/column streams; every
 * call gathers a fresh x through L2.  No reference counterpart: the
 * reference rebuilds ax for every new x (its conversion time).
 * ------------------------------------------------------------------------ */
typedef struct ispmv_plan_s *ispmv_plan;

/* Value storage of a plan.  Accumulation is FP64 in every form. */
#define ISPMV_VAL_F64 0      /* FP64 values (the drop-in) */
#define ISPMV_VAL_F32 1      /* FP32 values, FP32 multiply, FP64 accumulate */
#define ISPMV_VAL_F32_LO16 2 /* FP32 + BF16 residual lo-word on rows that need it */
/* Column storage of a plan. */
#define ISPMV_COL_U32 0      /* exact u32 columns */
#define ISPMV_COL_D16 1      /* 16-bit deltas from a per-unit base column */

/* Kernel variants a plan can run (ispmv_plan_opts.kernel). */
#define ISPMV_KERNEL_AUTO 0  /* the format's default */
#define ISPMV_KERNEL_LDG 1   /* slot-stream kernel, plain loads, register prefetch */
#define ISPMV_KERNEL_TMA 2   /* slot-stream kernel, 1D bulk copies (cp.async.bulk) into shared memory */
#define ISPMV_KERNEL_ROWS 3  /* row-parallel kernel (CSR: lanes per row; AXC: 8 lanes per row; K1) */
#define ISPMV_KERNEL_WIDE 4  /* slot-stream kernel over a lane-interleaved copy of the stream: 16 (or 8)
                                slots per lane; variants with a per-CTA x window in shared memory
                                (FP64/FP32 values, u32 columns), and plain-load variants that also
                                take 16-bit column deltas and BF16 lo-words */
#define ISPMV_VARIANT_QUEUE 16 /* slot-stream kernel as a work queue drained by persistent warps */

typedef struct {
  int val_kind;      /* ISPMV_VAL_* */
  int col_kind;      /* ISPMV_COL_* */
  int kernel;        /* ISPMV_KERNEL_* */
  int ctas_per_sm;   /* 0 = library default */
  int units_per_warp;/* work granule of one warp; 0 = library default */
  double lo_tol;     /* F32_LO16: rows whose FP32 rounding error bound exceeds
                        lo_tol relative carry a lo-word; 0 = default 1e-6 */
  int variant;       /* kernel variant (prefetch depth / register budget); 0 = default;
                        ISPMV_VARIANT_QUEUE = persistent warps pulling segments
                        from a device work queue */
  int rhs_block;     /* SpMM right-hand sides per pass: 8, 16 or 32; 0 = by k */
  int spmm_kernel;   /* SpMM: ISPMV_KERNEL_WIDE (four columns per lane, 32-byte X loads, the next
                        step's loads in flight while a step is consumed; k a multiple of 4, X and Y
                        32-byte aligned), ISPMV_KERNEL_LDG (two columns per lane) or
                        ISPMV_KERNEL_AUTO (WIDE for blocks of 16 or 32 columns where it applies,
                        else LDG) */
} ispmv_plan_opts;

void ispmv_plan_opts_default(ispmv_plan_opts *o);

/* Plans from host-built formats.  The host arrays are only read during the
 * call; the plan owns its device copies.  `csr` must have rl filled. */
int ispmv_plan_csr(const str_matCSR *csr, const ispmv_plan_opts *o, ispmv_plan *out);
int ispmv_plan_axc(const str_matCSR *csr, const str_matAXC *axc, const UIN *axi,
                   const ispmv_plan_opts *o, ispmv_plan *out);
/* reorder: 0 = int_k1 (result in chunk order, then orderArrayK1),
 *          1 = int_k1p (reordering integrated, scatter to y[permi]). */
int ispmv_plan_k1(const str_matCSR *csr, const str_matK1 *k1, int reorder,
                  const ispmv_plan_opts *o, ispmv_plan *out);
int ispmv_plan_axt(const str_matCSR *csr, const str_matAXT *axt, const UIN *axi,
                   const ispmv_plan_opts *o, ispmv_plan *out);
int ispmv_plan_destroy(ispmv_plan p);

/* A plan built on the GPU from a CSR matrix already in device memory, with
 * no host copy of the matrix.  It replaces the reference's host-side
 * conversion (getFormatDataAXT, intSpmv_main.c:1275-1381) for the compacted
 * AXT's slot stream (CSR order).  The arrays are bit for bit those
 * ispmv_plan_csr builds for the same matrix with kernel ISPMV_KERNEL_WIDE and
 * the same variant (per-CTA x windows included).  d_row (n+1), d_col and
 * d_val (nnz) are device pointers, read during the call.  Options: val_kind
 * F64 or F32, col_kind U32, kernel AUTO (the variant ispmv_plan_axt picks for
 * the compacted AXT) or WIDE; x-band and TMEM-staged variants give
 * ISPMV_ERR_UNSUPPORTED.  The matrix is checked on the device before use:
 * a decreasing row pointer, row[0] != 0, row[n] != nnz or a column >= n
 * gives ISPMV_ERR_ARG.  Synchronises `stream`. */
int ispmv_plan_dev_csr(UIN n, UIN nnz, const UIN *d_row, const UIN *d_col, const FPT *d_val,
                       const ispmv_plan_opts *o, ispmv_plan *out, void *stream);

/* The device arrays of a slot-stream plan with u32 columns (any stream
 * plan but the TMEM-staged ones), for checking one plan against another:
 * lengths, then copies into caller buffers (host or device; NULL skips an
 * array), synchronising `stream`.  val: slots_pad values of val_bytes each
 * (lane-interleaved when spl > 0), col: slots_pad, heads: slots_pad / 32
 * row-start words, segh: nseg, rowmap: nrowmap, empty: nempty; the per-CTA
 * x windows of the window variants: nwin starts (lo) and lengths (len).
 * No reference counterpart. */
typedef struct {
  uint64_t slots; uint64_t slots_pad; uint64_t seg_slots; uint64_t nseg;
  uint64_t nrowmap; uint64_t nempty; UIN val_bytes; UIN spl; uint64_t nwin;
} ispmv_plan_layout;
int ispmv_plan_get_layout(ispmv_plan p, ispmv_plan_layout *l);
int ispmv_plan_export_stream(ispmv_plan p, void *val, UIN *col, UIN *heads, UIN *segh, UIN *rowmap,
                             UIN *empty, void *stream);
int ispmv_plan_export_windows(ispmv_plan p, UIN *lo, UIN *len, void *stream);

/* y = A*x + beta*y with device pointers, beta in {0, 1}.  Stream-ordered.
 * A plan keeps per-product work areas on the device (segment records, the
 * FP32 copy of x of FP32-value plans): use one plan on one stream at a time;
 * products on two streams that overlap need two plans. */
int ispmv_plan_spmv(ispmv_plan p, const FPT *x, FPT *y, int beta, void *stream);
/* The same product as one CUDA-graph launch: the plan captures its kernels
 * (queue reset, SpMV, row fix-up) for this (x, y, beta) on first use, and
 * captures again when they change.  Stream-ordered on `stream`. */
int ispmv_plan_spmv_graph(ispmv_plan p, const FPT *x, FPT *y, int beta, void *stream);
/* Y = A*X for k right-hand sides, X and Y row-major (n x k), FP64.
 * ISPMV_ERR_UNSUPPORTED for spmm_kernel = ISPMV_KERNEL_WIDE when k is not a
 * multiple of 4 or X or Y is not 32-byte aligned. */
int ispmv_plan_spmm(ispmv_plan p, UIN k, const FPT *X, FPT *Y, void *stream);
/* End to end on HOST buffers: copies x in, runs the SpMV, copies y out and
 * synchronises `stream`.  Pinned host buffers give full PCIe bandwidth. */
int ispmv_plan_spmv_host(ispmv_plan p, const FPT *h_x, FPT *h_y, void *stream);

/* Status of the plan's last device work: ISPMV_ERR_TIMEOUT when a bounded
 * wait of a staged kernel gave up (the result is then invalid), else OK.
 * Synchronous (reads a device status word). */
int ispmv_plan_status(ispmv_plan p);

/* Kernel timing.  With pairs > 0 every ispmv_plan_spmv records a CUDA event
 * pair on its stream around the product's main kernel (not around the row
 * fix-up or K1's reorder that follow it), in a ring of `pairs` pairs;
 * pairs = 0 turns it off.  Graph launches record nothing.
 * ispmv_plan_kernel_ms returns the summed elapsed time of the recorded pairs
 * (at most `pairs`, the latest) and how many, then restarts the count; call
 * it after the stream is synchronised. */
int ispmv_plan_time_kernels(ispmv_plan p, int pairs);
int ispmv_plan_kernel_ms(ispmv_plan p, double *total_ms, int *launches);
/* The main kernel alone, timed: `reps` launches of the product's main kernel
 * (for FP32-value plans on the lane-interleaved kernel, with the rounding of
 * x to FP32 that precedes it) back to back on `stream` between one CUDA
 * event pair, without the row fix-up or K1's reorder; *ms = the mean per
 * launch.  Synchronises `stream`.  y is left without the fix-up's rows: an
 * ispmv_plan_spmv gives the product.  Unlike an event pair around each
 * launch, the timing holds no event record between consecutive launches. */
int ispmv_plan_time_main(ispmv_plan p, const FPT *x, FPT *y, int reps, void *stream, double *ms);
/* Name of the main kernel the plan's latest product launched (a static
 * string, "" before the first product), e.g. "stream_ldg<4,0,5>". */
const char *ispmv_plan_kernel_name(ispmv_plan p);

/* Plan facts: rows, nonzeros, value slots streamed, bytes of device
 * storage, and the algorithmic bytes of one SpMV:
 * nnz*(b_val + b_idx) + n*(b_x + b_y) + 4*(n+1). */
typedef struct {
  UIN nrows; UIN nnz; uint64_t slots; uint64_t device_bytes; double alg_bytes;
  int format; int val_kind; int col_kind; int kernel; UIN tile_h; UIN bs;
  char name[32];
} ispmv_plan_info;
int ispmv_plan_get_info(ispmv_plan p, ispmv_plan_info *info);

#endif /* !ISPMV_FPT_FLOAT: GPU format builders and plans are FP64 */

/* Library facts and diagnostics. */
const char *ispmv_version(void);
const char *ispmv_status_string(int status);
/* Last CUDA error text seen by the library on this thread ("" if none). */
const char *ispmv_last_error(void);
/* Kernel launches issued by the library since load (all ispmv_* calls). */
unsigned long long ispmv_launch_count(void);

/* Self-test of the bounded device wait the staged kernels use on their
 * mbarriers (no reference counterpart): waits on a barrier nothing completes,
 * and returns ISPMV_ERR_TIMEOUT when the wait gave up after its limit (about
 * 200 ms) as designed; *elapsed_ms = how long the wait took. */
int ispmv_selftest_bounded_wait(double *elapsed_ms, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* INTSPMV_H */
