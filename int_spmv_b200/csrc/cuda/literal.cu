// literal.cu - the reference's SpMV kernels as sm_100a kernels on the
// reference's own arrays (edoardoCB/int_spmv, intSpmv_main.c, "M:<line>").
//
// These take exactly the arrays the reference kernels take - including the
// x-baked `ax` of AXC and AXT, whose every 8 values are followed by the 8
// x[col] copies the builder stored (M:644, M:1171, M:1207, M:1247) - and
// keep each kernel's output contract: cf_CSR, int_axc and int_k1 overwrite
// their result, int_k1p scatters, the AXT kernels accumulate into y.
//
// Mapping (one warp = 32 lanes):
//   cf_CSR          8 lanes per row, shuffle reduction.
//   int_axc         8 lanes per row, lane k takes element k of every brick.
//   int_k1 / k1p    8 lanes per chunk (lane = row of the chunk): each column
//                   of a chunk is one coalesced 64-byte load of values.
//   int_axt_noc_h1  8 lanes per tile, 4 tiles per warp step; tile sums are
//                   combined per row with a segmented warp scan, so a row
//                   costs one atomic per warp instead of one per tile.
//   int_axt_noc     one warp per tile: lane = (sub-row group, column),
//                   columns reduced over sub-rows, then per-row runs of the
//                   8 columns combined before the atomics.
//   int_axt_com_h1  32 slots per warp step with a segmented scan; every slot
//                   carrying a descriptor, and every block start, opens a
//                   segment, so row-0 segments whose descriptor is 0 are
//                   summed (the reference skips them, M:1555) and segment
//                   sums are true sums, not prefix differences (M:1559).
//
// The file is compiled twice: with FPT = double (the reference's FP_DOUBLE
// build) and with ISPMV_FPT_FLOAT (FPT = float, every exported name gets
// the `_f32` suffix through intspmv.h).  Products and sums are FP64 in both;
// an FP32 result is rounded once when it is stored (or, for the AXT kernels,
// when each row run is added to y).
#include <cuda.h>

#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace ispmv {
namespace lit {

constexpr int TPB = 256;

__global__ void __launch_bounds__(TPB) k_cf_csr(UIN n, const UIN *__restrict__ row,
                                                const UIN *__restrict__ col,
                                                const FPT *__restrict__ val,
                                                const FPT *__restrict__ x, FPT *__restrict__ y) {
  const unsigned lane8 = threadIdx.x & 7u;
  const size_t r = ((size_t)blockIdx.x * TPB + threadIdx.x) >> 3;
  const bool live = r < n;
  double s = 0.0;
  if (live) {
    const UIN b = row[r], e = row[r + 1];
    for (UIN j = b + lane8; j < e; j += 8) s = fma((double)ld_stream(val + j), (double)ldg(x + ld_stream(col + j)), s);
  }
  s += __shfl_xor_sync(FULL, s, 4);
  s += __shfl_xor_sync(FULL, s, 2);
  s += __shfl_xor_sync(FULL, s, 1);
  if (live && lane8 == 0) y[r] = (FPT)s;
}

__global__ void __launch_bounds__(TPB) k_axc(UIN n, const FPT *__restrict__ ax,
                                             const UIN *__restrict__ brp, FPT *__restrict__ y) {
  const unsigned lane8 = threadIdx.x & 7u;
  const size_t r = ((size_t)blockIdx.x * TPB + threadIdx.x) >> 3;
  const bool live = r < n;
  double s = 0.0;
  if (live) {
    const UIN b = brp[r], e = brp[r + 1];
    for (UIN p = b; p < e; p += 16) s = fma((double)ld_stream(ax + p + lane8), (double)ld_stream(ax + p + 8 + lane8), s);
  }
  s += __shfl_xor_sync(FULL, s, 4);
  s += __shfl_xor_sync(FULL, s, 2);
  s += __shfl_xor_sync(FULL, s, 1);
  if (live && lane8 == 0) y[r] = (FPT)s;
}

// K1 (M:943-965) and K1 with integrated reordering (M:1026-1066).
template <bool SCATTER>
__global__ void __launch_bounds__(TPB) k_k1(UIN chunkNum, unsigned char mask, const FPT *__restrict__ val,
                                            const UIN *__restrict__ col, const UIN *__restrict__ chp,
                                            const UIN *__restrict__ nmc, const UIN *__restrict__ permi,
                                            const FPT *__restrict__ x, FPT *__restrict__ res) {
  const unsigned lane8 = threadIdx.x & 7u;
  const size_t c = ((size_t)blockIdx.x * TPB + threadIdx.x) >> 3;
  if (c >= chunkNum) return;
  const UIN off = chp[c], m = nmc[c];
  double s = 0.0;
  for (UIN k = 0; k < m; k++) {
    const size_t p = (size_t)off + (size_t)k * 8 + lane8;
    s = fma((double)ld_stream(val + p), (double)ldg(x + ld_stream(col + p)), s);
  }
  if (!SCATTER) {
    res[c * 8 + lane8] = (FPT)s;
  } else {
    const bool last = (c + 1 == chunkNum);
    if (!last || ((mask >> lane8) & 1u)) res[permi[c * 8 + lane8]] = (FPT)s;
  }
}

__global__ void k_order(UIN len, const UIN *__restrict__ permi, const FPT *__restrict__ dis,
                        FPT *__restrict__ ord) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < len) ord[permi[i]] = dis[i];
}

// AXT NOC tileH=1 (M:1385-1404): y[rwp[t]] += sum_k ax[16t+k] * ax[16t+8+k].
// Each warp covers STEPS*4 consecutive tiles.
constexpr int H1_STEPS = 8;
__global__ void __launch_bounds__(TPB) k_axt_noc_h1(UIN tileNum, const FPT *__restrict__ ax,
                                                    const UIN *__restrict__ rwp, FPT *__restrict__ y) {
  const unsigned lane = threadIdx.x & 31u, lane8 = lane & 7u;
  const size_t warp = ((size_t)blockIdx.x * TPB + threadIdx.x) >> 5;
  const size_t t0 = warp * (size_t)(H1_STEPS * 4);
  if (t0 >= tileNum) return;
  UIN crow = NO_ROW;
  double csum = 0.0;
  for (int st = 0; st < H1_STEPS; st++) {
    const size_t t = t0 + (size_t)st * 4 + (lane >> 3);
    const bool live = t < tileNum;
    double p = 0.0;
    UIN r = NO_ROW;
    if (live) {
      p = (double)ld_stream(ax + t * 16 + lane8) * (double)ld_stream(ax + t * 16 + 8 + lane8);
      r = rwp[t];
    }
    // within-tile sum (lane8 == 0 holds it)
    p += __shfl_xor_sync(FULL, p, 4);
    p += __shfl_xor_sync(FULL, p, 2);
    p += __shfl_xor_sync(FULL, p, 1);
    if (lane8) p = 0.0;
    const UIN rprev = __shfl_up_sync(FULL, r, 1);
    const bool head = (lane == 0) ? (r != crow) : (r != rprev);
    if (lane == 0) {
      if (!head) p += csum;
      else if (crow != NO_ROW) atomicAdd(y + crow, (FPT)csum);  // the carried run ended last step
    }
    const double s = warp_seg_scan(p, head);
    const UIN rnext = __shfl_down_sync(FULL, r, 1);
    if (lane < 31 && r != rnext && r != NO_ROW) atomicAdd(y + r, (FPT)s);
    crow = __shfl_sync(FULL, r, 31);
    csum = __shfl_sync(FULL, s, 31);
  }
  if (lane == 0 && crow != NO_ROW) atomicAdd(y + crow, (FPT)csum);
}

// AXT NOC tileH>1 (M:1443-1474): one warp per tile.
__global__ void __launch_bounds__(TPB) k_axt_noc(UIN tileNum, UIN th, const FPT *__restrict__ ax,
                                                 const UIN *__restrict__ rwp, FPT *__restrict__ y) {
  const unsigned lane = threadIdx.x & 31u, c = lane & 7u;
  const size_t t = ((size_t)blockIdx.x * TPB + threadIdx.x) >> 5;
  if (t >= tileNum) return;
  const FPT *tile = ax + t * (size_t)th * 16;
  double s = 0.0;
  for (UIN R = lane >> 3; R < th; R += 4)
    s = fma((double)ld_stream(tile + R * 16 + c), (double)ld_stream(tile + R * 16 + 8 + c), s);
  s += __shfl_xor_sync(FULL, s, 8);
  s += __shfl_xor_sync(FULL, s, 16);
  // lanes 0..7 hold the 8 column sums; combine runs of equal rows
  const UIN r = (lane < 8) ? rwp[t * 8 + c] : NO_ROW;
  const UIN rprev = __shfl_up_sync(FULL, r, 1);
  const bool head = (lane == 0) || (r != rprev);
  const double v = warp_seg_scan(lane < 8 ? s : 0.0, head);
  const UIN rnext = __shfl_down_sync(FULL, r, 1);
  if (lane < 8 && r != rnext) atomicAdd(y + r, (FPT)v);
}

// AXT COM tileH=1 (M:1517-1566), true segmented sums.
constexpr int COM_STEPS = 16;
__global__ void __launch_bounds__(TPB) k_axt_com_h1(UIN bs, UIN lg, UIN lenRWP, const FPT *__restrict__ ax,
                                                    const UIN *__restrict__ rwp, FPT *__restrict__ y) {
  const unsigned lane = threadIdx.x & 31u;
  const size_t warp = ((size_t)blockIdx.x * TPB + threadIdx.x) >> 5;
  const size_t p0 = warp * (size_t)(COM_STEPS * 32);
  if (p0 >= lenRWP) return;
  UIN crow = NO_ROW;
  double csum = 0.0;
  for (int st = 0; st < COM_STEPS; st++) {
    const size_t p = p0 + (size_t)st * 32 + lane;
    const bool live = p < lenRWP;
    double v = 0.0;
    bool head = false;
    UIN hrow = 0;
    if (live) {
      const size_t a = (p >> 3) * 16 + (p & 7);
      v = (double)ld_stream(ax + a) * (double)ld_stream(ax + a + 8);
      const UIN d = rwp[p];
      head = (d != 0) || ((p & (bs - 1)) == 0);
      hrow = d >> lg;
    }
    // row of each lane's run: the row of the latest head at or before it
    int hl = head ? (int)lane : -1;
#pragma unroll
    for (unsigned d = 1; d < 32; d <<= 1) {
      const int u = __shfl_up_sync(FULL, hl, d);
      if (lane >= d) hl = max(hl, u);
    }
    const UIN hr = __shfl_sync(FULL, hrow, hl < 0 ? 0 : hl);
    const UIN r = live ? (hl < 0 ? crow : hr) : NO_ROW;
    const bool seg = (lane == 0) ? (head || r != crow) : (head || !live);
    if (lane == 0) {
      if (!seg) v += csum;
      else if (crow != NO_ROW) atomicAdd(y + crow, (FPT)csum);  // the carried run ended last step
    }
    const double s = warp_seg_scan(v, seg);
    const bool nexthead = __shfl_down_sync(FULL, (unsigned)(head || !live), 1) != 0;
    if (lane < 31 && live && nexthead && r != NO_ROW) atomicAdd(y + r, (FPT)s);
    crow = __shfl_sync(FULL, r, 31);
    csum = __shfl_sync(FULL, s, 31);
  }
  if (lane == 0 && crow != NO_ROW) atomicAdd(y + crow, (FPT)csum);
}

inline unsigned blocks_for(size_t threads) { return (unsigned)((threads + TPB - 1) / TPB); }

}  // namespace lit
}  // namespace ispmv

using namespace ispmv;

ISPMV_API int ispmv_dev_cf_csr(UIN nrows, const UIN *row, const UIN *col, const FPT *val, const FPT *vec,
                               FPT *res, void *stream) {
  if (nrows == 0) return ISPMV_OK;
  if (!row || !res || !vec) return ISPMV_ERR_ARG;
  lit::k_cf_csr<<<lit::blocks_for((size_t)nrows * 8), lit::TPB, 0, as_stream(stream)>>>(nrows, row, col, val, vec, res);
  return check_launch("ispmv_dev_cf_csr");
}

ISPMV_API int ispmv_dev_int_axc(UIN nrows, const FPT *ax, const UIN *brp, FPT *y, void *stream) {
  if (nrows == 0) return ISPMV_OK;
  if (!ax || !brp || !y) return ISPMV_ERR_ARG;
  lit::k_axc<<<lit::blocks_for((size_t)nrows * 8), lit::TPB, 0, as_stream(stream)>>>(nrows, ax, brp, y);
  return check_launch("ispmv_dev_int_axc");
}

ISPMV_API int ispmv_dev_int_k1(UIN chunkNum, const FPT *val, const UIN *col, const UIN *chp, const UIN *nmc,
                               const FPT *vec, FPT *res, void *stream) {
  if (chunkNum == 0) return ISPMV_OK;
  if (!val || !col || !chp || !nmc || !vec || !res) return ISPMV_ERR_ARG;
  lit::k_k1<false><<<lit::blocks_for((size_t)chunkNum * 8), lit::TPB, 0, as_stream(stream)>>>(
      chunkNum, 0xFF, val, col, chp, nmc, nullptr, vec, res);
  return check_launch("ispmv_dev_int_k1");
}

ISPMV_API int ispmv_dev_order_k1(UIN len, const UIN *permi, const FPT *arrDis, FPT *arrOrd, void *stream) {
  if (len == 0) return ISPMV_OK;
  if (!permi || !arrDis || !arrOrd) return ISPMV_ERR_ARG;
  lit::k_order<<<lit::blocks_for(len), lit::TPB, 0, as_stream(stream)>>>(len, permi, arrDis, arrOrd);
  return check_launch("ispmv_dev_order_k1");
}

ISPMV_API int ispmv_dev_int_k1p(unsigned char mask, UIN chunkNum, const FPT *val, const UIN *col, const UIN *chp,
                                const UIN *nmc, const UIN *permi, const FPT *vec, FPT *res, void *stream) {
  if (chunkNum == 0) return ISPMV_OK;
  if (!val || !col || !chp || !nmc || !permi || !vec || !res) return ISPMV_ERR_ARG;
  lit::k_k1<true><<<lit::blocks_for((size_t)chunkNum * 8), lit::TPB, 0, as_stream(stream)>>>(
      chunkNum, mask, val, col, chp, nmc, permi, vec, res);
  return check_launch("ispmv_dev_int_k1p");
}

ISPMV_API int ispmv_dev_int_axt_noc_h1(UIN tileNum, const FPT *ax, const UIN *rwp, FPT *y, void *stream) {
  if (tileNum == 0) return ISPMV_OK;
  if (!ax || !rwp || !y) return ISPMV_ERR_ARG;
  const size_t warps = ((size_t)tileNum + lit::H1_STEPS * 4 - 1) / (lit::H1_STEPS * 4);
  lit::k_axt_noc_h1<<<lit::blocks_for(warps * 32), lit::TPB, 0, as_stream(stream)>>>(tileNum, ax, rwp, y);
  return check_launch("ispmv_dev_int_axt_noc_h1");
}

ISPMV_API int ispmv_dev_int_axt_noc(UIN tileNum, UIN tileHeight, const FPT *ax, const UIN *rwp, FPT *y,
                                   void *stream) {
  if (tileNum == 0) return ISPMV_OK;
  if (!ax || !rwp || !y || tileHeight == 0) return ISPMV_ERR_ARG;
  lit::k_axt_noc<<<lit::blocks_for((size_t)tileNum * 32), lit::TPB, 0, as_stream(stream)>>>(tileNum, tileHeight, ax,
                                                                                            rwp, y);
  return check_launch("ispmv_dev_int_axt_noc");
}

ISPMV_API int ispmv_dev_int_axt_com_h1(UIN bn, UIN bs, UIN log, UIN thw, UIN tn, UIN lenAX, UIN lenRWP,
                                       const FPT *ax, const UIN *rwp, FPT *y, void *stream) {
  if (thw != 8) return ISPMV_ERR_UNSUPPORTED;
  // bs <= 512 also makes every warp's first slot (a multiple of 512) a block start
  if (bs < 8 || bs > 512 || (bs & (bs - 1)) || (1u << log) != bs) return ISPMV_ERR_ARG;
  if ((uint64_t)tn * 8 != lenRWP || (uint64_t)tn * 16 != lenAX || (uint64_t)bn * bs < lenRWP) return ISPMV_ERR_ARG;
  if (lenRWP == 0) return ISPMV_OK;
  if (!ax || !rwp || !y) return ISPMV_ERR_ARG;
  const size_t warps = ((size_t)lenRWP + lit::COM_STEPS * 32 - 1) / (lit::COM_STEPS * 32);
  lit::k_axt_com_h1<<<lit::blocks_for(warps * 32), lit::TPB, 0, as_stream(stream)>>>(bs, log, lenRWP, ax, rwp, y);
  return check_launch("ispmv_dev_int_axt_com_h1");
}

#ifndef ISPMV_FPT_FLOAT  // FP64 only
// ---------------------------------------------------------------------------
// K1 product in original row order that allocates nothing.  The chunk-order
// result of the K1 kernel (the `res` array int_k1 hands to orderArrayK1)
// lives in this file-scope device array instead of caller or library
// allocations; every GPU that loads the library holds it (8 MiB) until exit.
static __device__ __align__(256) double g_k1_rows[ISPMV_K1_NOALLOC_MAX_ROWS];

namespace {
// The array's device address, per device, with the id of the context it was
// looked up in.  A context that is destroyed and created again (for one,
// after cudaDeviceReset) loads the module afresh, possibly at another
// address, and gets a new id: the address is then looked up again.
struct K1RowsAddr {
  unsigned long long ctx_id;
  double *addr;
};
std::mutex g_k1_rows_mu;
K1RowsAddr g_k1_rows_addr[64] = {};

// cuCtxGetCurrent / cuCtxGetId through the runtime's driver entry points, so
// the library links no driver library.  Null when unavailable.
typedef CUresult(CUDAAPI *CtxGetCurrentFn)(CUcontext *);
typedef CUresult(CUDAAPI *CtxGetIdFn)(CUcontext, unsigned long long *);
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;
std::once_flag g_ctx_fns_once;

void find_ctx_fns() {
  void *f = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
    g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(f);
  f = nullptr;
  if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
    g_ctx_id = reinterpret_cast<CtxGetIdFn>(f);
  (void)cudaGetLastError();
}

// Id of the calling thread's current context; 0 when there is none yet or
// the driver entry points are unavailable.
unsigned long long current_ctx_id() {
  std::call_once(g_ctx_fns_once, find_ctx_fns);
  if (!g_ctx_current || !g_ctx_id) return 0;
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (g_ctx_current(&c) != CUDA_SUCCESS || !c) return 0;
  if (g_ctx_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// The array's address in the current context (the host-side symbol is not a
// device address).  Looked up with cudaGetSymbolAddress the first time a
// context of this device calls, then reused while that context lives; with
// no context id available it is looked up on every call.
int k1_rows_scratch(double **out) {
  int dev = 0;
  ISPMV_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(ISPMV_ERR_UNSUPPORTED, "ispmv_dev_k1_spmv_noalloc: device index >= 64");
  std::lock_guard<std::mutex> g(g_k1_rows_mu);
  K1RowsAddr &c = g_k1_rows_addr[dev];
  const unsigned long long id = current_ctx_id();
  if (!c.addr || id == 0 || id != c.ctx_id) {
    void *addr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&addr, g_k1_rows);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_k1_rows)");
    c.addr = static_cast<double *>(addr);
    c.ctx_id = current_ctx_id();  // the lookup makes the device's context current if none was
  }
  *out = c.addr;
  return ISPMV_OK;
}
}  // namespace

ISPMV_API int ispmv_dev_k1_spmv_noalloc(UIN nrows, UIN chunkNum, const FPT *val, const UIN *col, const UIN *chp,
                                        const UIN *nmc, const UIN *permi, const FPT *vec, FPT *y, void *stream) {
  if (nrows == 0) return ISPMV_OK;
  if (!val || !col || !chp || !nmc || !permi || !vec || !y)
    return fail(ISPMV_ERR_ARG, "ispmv_dev_k1_spmv_noalloc: null array");
  if ((uint64_t)chunkNum * 8 < nrows || (uint64_t)chunkNum * 8 >= (uint64_t)nrows + 8)
    return fail(ISPMV_ERR_ARG, "ispmv_dev_k1_spmv_noalloc: chunkNum must be ceil(nrows / 8)");
  if ((uint64_t)chunkNum * 8 > ISPMV_K1_NOALLOC_MAX_ROWS)
    return fail(ISPMV_ERR_ARG, "ispmv_dev_k1_spmv_noalloc: more than ISPMV_K1_NOALLOC_MAX_ROWS (1048576) rows");
  double *res = nullptr;
  int st = k1_rows_scratch(&res);
  if (st) return st;
  // the K1 kernel writes all chunkNum*8 entries of res before the reorder
  // reads any, so nothing left by an earlier call is ever read
  lit::k_k1<false><<<lit::blocks_for((size_t)chunkNum * 8), lit::TPB, 0, as_stream(stream)>>>(
      chunkNum, 0xFF, val, col, chp, nmc, nullptr, vec, res);
  st = check_launch("ispmv_dev_k1_spmv_noalloc (chunks)");
  if (st) return st;
  lit::k_order<<<lit::blocks_for(nrows), lit::TPB, 0, as_stream(stream)>>>(nrows, permi, res, y);
  return check_launch("ispmv_dev_k1_spmv_noalloc (reorder)");
}

#endif  // !ISPMV_FPT_FLOAT

// ---------------------------------------------------------------------------
// Host-pointer forms with the reference's names.  A small grow-only pool of
// device buffers per process keeps repeated calls from re-allocating.
namespace {
std::mutex g_pool_mu;
std::vector<std::pair<void *, size_t>> g_pool(8, {nullptr, 0});

int pool_get(int slot, size_t bytes, void **out) {
  auto &b = g_pool[slot];
  if (b.second < bytes) {
    if (b.first) cudaFree(b.first);
    b = {nullptr, 0};
    void *p = nullptr;
    ISPMV_TRY(cudaMalloc(&p, bytes ? bytes : 16));
    b = {p, bytes};
  }
  *out = b.first;
  return ISPMV_OK;
}

[[noreturn]] void die(const char *fn, int st) {
  fflush(stdout);
  printf("\n%s failed: %s (%s)\n", fn, ispmv_status_string(st), ispmv_last_error());
  fflush(stdout);
  exit(EXIT_FAILURE);
}

template <typename T>
int up(int slot, const T *h, size_t n, T **d) {
  void *p;
  int st = pool_get(slot, n * sizeof(T), &p);
  if (st) return st;
  if (n) ISPMV_TRY(cudaMemcpy(p, h, n * sizeof(T), cudaMemcpyHostToDevice));
  *d = (T *)p;
  return ISPMV_OK;
}
template <typename T>
int down(T *h, const T *d, size_t n) {
  if (n) ISPMV_TRY(cudaMemcpy(h, d, n * sizeof(T), cudaMemcpyDeviceToHost));
  return ISPMV_OK;
}
#define CHK(expr)             \
  do {                        \
    int s__ = (expr);         \
    if (s__) die(FN, s__);    \
  } while (0)
}  // namespace

ISPMV_API void cf_CSR(const str_matCSR m, const FPT *vec, FPT *res) {
  static const char *FN = "cf_CSR";
  std::lock_guard<std::mutex> g(g_pool_mu);
  UIN *row, *col;
  FPT *val, *x, *y;
  CHK(up(0, m.row, (size_t)m.nrows + 1, &row));
  CHK(up(1, m.col, m.nnz, &col));
  CHK(up(2, m.val, m.nnz, &val));
  CHK(up(3, vec, m.nrows, &x));
  CHK(pool_get(4, (size_t)m.nrows * sizeof(FPT), (void **)&y));
  CHK(ispmv_dev_cf_csr(m.nrows, row, col, val, x, y, nullptr));
  CHK(down(res, y, m.nrows));
}

ISPMV_API void int_axc(const UIN ompNT, const UIN nrows, const FPT *ax, const UIN *brp, FPT *y) {
  static const char *FN = "int_axc";
  (void)ompNT;
  std::lock_guard<std::mutex> g(g_pool_mu);
  UIN *dbrp;
  FPT *dax, *dy;
  CHK(up(0, brp, (size_t)nrows + 1, &dbrp));
  UIN lenAX = nrows ? brp[nrows] : 0;
  CHK(up(1, ax, lenAX, &dax));
  CHK(pool_get(2, (size_t)nrows * sizeof(FPT), (void **)&dy));
  CHK(ispmv_dev_int_axc(nrows, dax, dbrp, dy, nullptr));
  CHK(down(y, dy, nrows));
}

// The K1 arrays' lengths follow from chp/nmc (lenVC = chp[last] + 8*nmc[last]).
static size_t k1_len(UIN chunkNum, const UIN *chp, const UIN *nmc) {
  return chunkNum ? (size_t)chp[chunkNum - 1] + (size_t)8 * nmc[chunkNum - 1] : 0;
}
// x is indexed by column, and K1 columns are < nrows <= chunkNum*8.
ISPMV_API void int_k1(const UIN ompNT, const UIN chunkNum, const FPT *val, const UIN *col, const UIN *chp,
                      const UIN *nmc, const FPT *vec, FPT *res) {
  static const char *FN = "int_k1";
  (void)ompNT;
  std::lock_guard<std::mutex> g(g_pool_mu);
  const size_t len = k1_len(chunkNum, chp, nmc);
  UIN *dcol, *dchp, *dnmc;
  FPT *dval, *dx, *dres;
  UIN maxc = 0;
  for (size_t i = 0; i < len; i++) maxc = col[i] > maxc ? col[i] : maxc;
  CHK(up(0, val, len, &dval));
  CHK(up(1, col, len, &dcol));
  CHK(up(2, chp, chunkNum, &dchp));
  CHK(up(3, nmc, chunkNum, &dnmc));
  CHK(up(4, vec, len ? (size_t)maxc + 1 : 0, &dx));
  CHK(pool_get(5, (size_t)chunkNum * 8 * sizeof(FPT), (void **)&dres));
  CHK(ispmv_dev_int_k1(chunkNum, dval, dcol, dchp, dnmc, dx, dres, nullptr));
  CHK(down(res, dres, (size_t)chunkNum * 8));
}

ISPMV_API void orderArrayK1(const UIN ompNT, const UIN len, const UIN *permi, const FPT *arrDis, FPT *arrOrd) {
  static const char *FN = "orderArrayK1";
  (void)ompNT;
  std::lock_guard<std::mutex> g(g_pool_mu);
  UIN *dp;
  FPT *dd, *dord;
  CHK(up(0, permi, len, &dp));
  CHK(up(1, arrDis, len, &dd));
  CHK(up(2, arrOrd, len, &dord));  // rows outside permi keep their values
  CHK(ispmv_dev_order_k1(len, dp, dd, dord, nullptr));
  CHK(down(arrOrd, dord, len));
}

ISPMV_API void int_k1p(const UIN ompNT, const unsigned char mask, const UIN chunkNum, const FPT *val, const UIN *col,
                       const UIN *chp, const UIN *nmc, const UIN *permi, const FPT *vec, FPT *res) {
  static const char *FN = "int_k1p";
  (void)ompNT;
  std::lock_guard<std::mutex> g(g_pool_mu);
  const size_t len = k1_len(chunkNum, chp, nmc);
  // rows = chunkNum*8 minus the masked-off tail lanes
  unsigned live = 0;
  for (unsigned i = 0; i < 8; i++) live += (mask >> i) & 1u;
  const size_t n = chunkNum ? (size_t)(chunkNum - 1) * 8 + live : 0;
  UIN *dcol, *dchp, *dnmc, *dp;
  FPT *dval, *dx, *dres;
  CHK(up(0, val, len, &dval));
  CHK(up(1, col, len, &dcol));
  CHK(up(2, chp, chunkNum, &dchp));
  CHK(up(3, nmc, chunkNum, &dnmc));
  CHK(up(4, permi, (size_t)chunkNum * 8, &dp));
  CHK(up(5, vec, n, &dx));
  CHK(up(6, res, n, &dres));
  CHK(ispmv_dev_int_k1p(mask, chunkNum, dval, dcol, dchp, dnmc, dp, dx, dres, nullptr));
  CHK(down(res, dres, n));
}

// The AXT kernels accumulate into y, whose length the signature does not
// carry: it is 1 + the largest row id in rwp.
static size_t axt_rows(const UIN *rwp, size_t len, UIN lg) {
  UIN m = 0;
  for (size_t i = 0; i < len; i++) m = (rwp[i] >> lg) > m ? (rwp[i] >> lg) : m;
  return len ? (size_t)m + 1 : 0;
}

ISPMV_API void int_axt_noc_h1(const UIN ompNT, const UIN tileNum, const FPT *ax, const UIN *rwp, FPT *y) {
  static const char *FN = "int_axt_noc_h1";
  (void)ompNT;
  std::lock_guard<std::mutex> g(g_pool_mu);
  const size_t n = axt_rows(rwp, tileNum, 0);
  FPT *dax, *dy;
  UIN *drwp;
  CHK(up(0, ax, (size_t)tileNum * 16, &dax));
  CHK(up(1, rwp, tileNum, &drwp));
  CHK(up(2, y, n, &dy));
  CHK(ispmv_dev_int_axt_noc_h1(tileNum, dax, drwp, dy, nullptr));
  CHK(down(y, dy, n));
}

ISPMV_API void int_axt_noc(const UIN ompNT, const UIN tileNum, const UIN tileHeight, const FPT *ax, const UIN *rwp,
                           FPT *y) {
  static const char *FN = "int_axt_noc";
  (void)ompNT;
  std::lock_guard<std::mutex> g(g_pool_mu);
  const size_t n = axt_rows(rwp, (size_t)tileNum * 8, 0);
  FPT *dax, *dy;
  UIN *drwp;
  CHK(up(0, ax, (size_t)tileNum * 16 * tileHeight, &dax));
  CHK(up(1, rwp, (size_t)tileNum * 8, &drwp));
  CHK(up(2, y, n, &dy));
  CHK(ispmv_dev_int_axt_noc(tileNum, tileHeight, dax, drwp, dy, nullptr));
  CHK(down(y, dy, n));
}

ISPMV_API void int_axt_com_h1(const UIN ompNT, const UIN bn, const UIN bs, const UIN log, const UIN thw, const UIN tn,
                              const UIN lenAX, const UIN lenRWP, const FPT *ax, const UIN *rwp, FPT *y) {
  static const char *FN = "int_axt_com_h1";
  (void)ompNT;
  std::lock_guard<std::mutex> g(g_pool_mu);
  const size_t n = axt_rows(rwp, lenRWP, log);
  FPT *dax, *dy;
  UIN *drwp;
  CHK(up(0, ax, lenAX, &dax));
  CHK(up(1, rwp, lenRWP, &drwp));
  CHK(up(2, y, n, &dy));
  CHK(ispmv_dev_int_axt_com_h1(bn, bs, log, thw, tn, lenAX, lenRWP, dax, drwp, dy, nullptr));
  CHK(down(y, dy, n));
}
