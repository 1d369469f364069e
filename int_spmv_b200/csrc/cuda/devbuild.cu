// devbuild.cu - format conversion on the GPU: the AXT arrays that
// getFormatDataAXT builds on the host (M:1275-1381) - con, the x-baked ax
// and sec - built from a CSR matrix and an x already in device memory.
//
// The layout rules are the host builder's (builders.c), in closed form:
// a running slot count s over rows (each row padded to a multiple of 8 for
// tileH = 1 or of tileH above it in NOC mode, packed in COM mode); slot s
// sits in tile T = s/(8*th), column (s/th)%8, sub-row s%th, i.e. at
// ax[T*16*th + (s%th)*16 + (s/th)%8] with its x copy 8 further; con[r] is
// that position for the row's first slot; sec holds the row of each tile
// (NOC, th = 1) or tile column (NOC, th > 1), or the COM segment descriptor
// (row << log2 bs) | min(left - 1, bs - 1 - s%bs) at row and block starts.
// Padding is zero.  The arrays are bit-identical to the host builder's.
//
// Steps: row slot counts -> exclusive prefix (three scan kernels over u64)
// -> sizes read back to the host (one synchronisation, to allocate) ->
// one warp per row writes its slots.
//
// The K1 arrays of getFormatDataK1 (M:841-905) likewise: rows sorted by
// length, descending, equal lengths in ascending row order (the order of the
// reference's qsort, M:775-796) by a stable radix sort (CUB, builder only);
// nmc[c] = the length of chunk c's first row, chp = the exclusive prefix of
// 8*nmc; val/col column-major per chunk, zero padding.
#include <algorithm>
#include <cstdio>
#include <cstring>

#include <cub/device/device_radix_sort.cuh>

#include "common.cuh"

using namespace ispmv;

namespace {

constexpr int ST = 1024;        // threads per scan block
constexpr int SI = 4;           // items per thread
constexpr int SB = ST * SI;     // items per scan block

__global__ void row_slots(UIN n, const UIN *__restrict__ row, UIN grp, int noc, uint64_t *__restrict__ cnt) {
  const size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r > n) return;
  if (r == n) {
    cnt[n] = 0;  // the scan's last entry becomes the total
    return;
  }
  const uint64_t l = row[r + 1] - row[r];
  cnt[r] = noc ? (l + grp - 1) / grp * grp : l;
}

// Exclusive prefix of one block's SB items; bsum[b] = the block's total.
__global__ void __launch_bounds__(ST) scan_block(size_t len, const uint64_t *__restrict__ in,
                                                 uint64_t *__restrict__ out, uint64_t *__restrict__ bsum) {
  __shared__ uint64_t wsum[ST / 32];
  const size_t base = (size_t)blockIdx.x * SB + (size_t)threadIdx.x * SI;
  uint64_t v[SI], t = 0;
#pragma unroll
  for (int i = 0; i < SI; i++) {
    v[i] = base + i < len ? in[base + i] : 0;
    t += v[i];
  }
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  uint64_t incl = t;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint64_t u = __shfl_up_sync(FULL, incl, d);
    if ((int)lane >= d) incl += u;
  }
  if (lane == 31) wsum[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    uint64_t w = lane < ST / 32 ? wsum[lane] : 0, wi = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint64_t u = __shfl_up_sync(FULL, wi, d);
      if ((int)lane >= d) wi += u;
    }
    if (lane < ST / 32) wsum[lane] = wi - w;  // exclusive over warps
    if (lane == 31) bsum[blockIdx.x] = wi;
  }
  __syncthreads();
  uint64_t run = wsum[wid] + incl - t;
#pragma unroll
  for (int i = 0; i < SI; i++) {
    if (base + i < len) out[base + i] = run;
    run += v[i];
  }
}

// Exclusive prefix of the nb block totals in place (one block, any nb).
__global__ void __launch_bounds__(ST) scan_totals(size_t nb, uint64_t *__restrict__ bsum) {
  __shared__ uint64_t wsum[ST / 32];
  __shared__ uint64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  for (size_t c0 = 0; c0 < nb; c0 += ST) {
    const size_t i = c0 + threadIdx.x;
    const uint64_t v = i < nb ? bsum[i] : 0;
    uint64_t incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint64_t u = __shfl_up_sync(FULL, incl, d);
      if ((int)lane >= d) incl += u;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      uint64_t w = lane < ST / 32 ? wsum[lane] : 0, wi = w;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint64_t u = __shfl_up_sync(FULL, wi, d);
        if ((int)lane >= d) wi += u;
      }
      if (lane < ST / 32) wsum[lane] = wi - w;
    }
    __syncthreads();
    const uint64_t c = carry;
    if (i < nb) bsum[i] = c + wsum[wid] + incl - v;
    __syncthreads();
    if (threadIdx.x == ST - 1) carry = c + wsum[wid] + incl;
    __syncthreads();
  }
}

__global__ void add_block_offsets(size_t len, uint64_t *__restrict__ out, const uint64_t *__restrict__ bsum) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < len) out[i] += bsum[i / SB];
}

// Slot s's value position in ax.  lenAX < 2^32 (checked before the fill),
// so slots and positions fit in 32 bits.
__device__ __forceinline__ UIN axt_pos(UIN s, UIN thw, UIN th) {
  const UIN ths = thw * th;
  const UIN T = s / ths, w = s - T * ths;
  return T * 2 * ths + (w % th) * 2 * thw + w / th;
}

// One warp per row: con, the row's values and x copies, and sec.
__global__ void __launch_bounds__(256) fill_axt(UIN n, const UIN *__restrict__ row, const UIN *__restrict__ col,
                                                const FPT *__restrict__ val, const FPT *__restrict__ x,
                                                const uint64_t *__restrict__ off, UIN thw, UIN th, int noc, UIN bs,
                                                UIN lg, UIN *__restrict__ con, FPT *__restrict__ ax,
                                                UIN *__restrict__ sec) {
  const size_t r = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (r >= n) return;
  const UIN s0 = (UIN)off[r];
  if (lane == 0) con[r] = axt_pos(s0, thw, th);
  const UIN j0 = row[r], len = row[r + 1] - j0;
  for (UIN k = lane; k < len; k += 32) {
    const UIN s = s0 + k;
    const UIN p = axt_pos(s, thw, th);
    ax[p] = val[j0 + k];
    ax[p + thw] = x[col[j0 + k]];
    if (noc) {
      const UIN T = s / (thw * th);
      sec[th == 1 ? T : T * thw + (s / th) % thw] = (UIN)r;
    } else if (k == 0 || (s & (bs - 1)) == 0) {
      const UIN q1 = len - k - 1, q2 = bs - 1 - (s & (bs - 1));
      sec[s] = ((UIN)r << lg) | (q1 > q2 ? q2 : q1);
    }
  }
}

__global__ void row_lengths(UIN n, const UIN *__restrict__ row, UIN *__restrict__ rl, UIN *__restrict__ ids) {
  const size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  rl[r] = row[r + 1] - row[r];
  ids[r] = (UIN)r;
}

// chunk c: nmc = its first row's length; cnt = 8*nmc (scanned into chp)
__global__ void chunk_widths(UIN cn, const UIN *__restrict__ rl_sorted, UIN *__restrict__ nmc,
                             uint64_t *__restrict__ cnt) {
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c > cn) return;
  if (c == cn) {
    cnt[cn] = 0;
    return;
  }
  nmc[c] = rl_sorted[c * 8];
  cnt[c] = 8ull * rl_sorted[c * 8];
}

// One thread per (chunk, lane): the row's elements go down the chunk column.
__global__ void fill_k1(UIN n, const UIN *__restrict__ row, const UIN *__restrict__ col, const FPT *__restrict__ val,
                        const UIN *__restrict__ permi, const uint64_t *__restrict__ chp64, UIN *__restrict__ chp,
                        FPT *__restrict__ kval, UIN *__restrict__ kcol) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t c = i / 8, lane = i % 8;
  const UIN base = (UIN)chp64[c];
  if (lane == 0) chp[c] = base;
  const UIN r = permi[i], j0 = row[r], len = row[r + 1] - j0;
  for (UIN k = 0; k < len; k++) {
    const size_t p = (size_t)base + (size_t)k * 8 + lane;
    kval[p] = val[j0 + k];
    kcol[p] = col[j0 + k];
  }
}

UIN floor_log2_lt1024(UIN v) {  // M:1286-1287 / M:1341-1348: the largest i < 10 with (v >> i) == 1
  UIN r = 0;
  for (UIN i = 0; i < 10; i++)
    if ((v >> i) == 1) r = i;
  return r;
}

}  // namespace

// Copies a device-built AXT's con/ax/sec into caller buffers (host or
// device memory; NULL skips an array) and synchronises `stream`.
ISPMV_API int ispmv_dev_axt_export(const str_matAXT *m, UIN *con, FPT *ax, UIN *sec, void *stream) {
  if (!m) return ISPMV_ERR_ARG;
  cudaStream_t s = as_stream(stream);
  if (con && m->lenCON) ISPMV_TRY(cudaMemcpyAsync(con, m->con, (size_t)m->lenCON * sizeof(UIN), cudaMemcpyDefault, s));
  if (ax && m->lenAX) ISPMV_TRY(cudaMemcpyAsync(ax, m->ax, (size_t)m->lenAX * sizeof(FPT), cudaMemcpyDefault, s));
  if (sec && m->lenSEC) ISPMV_TRY(cudaMemcpyAsync(sec, m->sec, (size_t)m->lenSEC * sizeof(UIN), cudaMemcpyDefault, s));
  ISPMV_TRY(cudaStreamSynchronize(s));
  return ISPMV_OK;
}

ISPMV_API int ispmv_dev_axt_free(str_matAXT *m) {
  if (!m) return ISPMV_ERR_ARG;
  cudaFree(m->con);
  cudaFree(m->ax);
  cudaFree(m->sec);
  std::memset(m, 0, sizeof *m);
  return ISPMV_OK;
}

// getFormatDataAXT on the GPU.  d_row (n+1), d_col, d_val (nnz) and d_x (n)
// are device pointers; the struct's con/ax/sec come back as device
// pointers (free with ispmv_dev_axt_free); fd->ct is the GPU time of the
// conversion in seconds (CUDA events on `stream`; the call synchronises it).
ISPMV_API int ispmv_dev_build_axt(UIN bs, UIN thw, UIN th, const char *mode, UIN n, UIN nnz, const UIN *d_row,
                                  const UIN *d_col, const FPT *d_val, const FPT *d_x, str_matAXT *m,
                                  str_formatData *fd, void *stream) {
  if (!m || !mode || !d_row || !d_x || n == 0 || (nnz && (!d_col || !d_val))) return ISPMV_ERR_ARG;
  if (thw != 8 || th == 0) return thw == 0 || th == 0 ? ISPMV_ERR_ARG : ISPMV_ERR_UNSUPPORTED;
  const int noc = std::strcmp(mode, "NOC") == 0, com = std::strcmp(mode, "COM") == 0;
  if (!noc && !com) return ISPMV_ERR_ARG;
  if (com && th != 1) return ISPMV_ERR_UNSUPPORTED;  // unimplemented in the reference, M:1338-1362
  UIN lg = 0;
  if (com) {
    if (bs < 2 || bs > 512 || (bs & (bs - 1))) return ISPMV_ERR_ARG;
    lg = floor_log2_lt1024(bs);
    if (((uint64_t)(n - 1) << lg) > 0xFFFFFFFFull) return ISPMV_ERR_OVERFLOW;  // row << log
  }
  cudaStream_t s = as_stream(stream);
  std::memset(m, 0, sizeof *m);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  uint64_t *cnt = nullptr, *off = nullptr, *bsum = nullptr;
  int st = ISPMV_OK;
  const size_t len = (size_t)n + 1, nb = (len + SB - 1) / SB;
  const UIN grp = th == 1 ? thw : th;
  uint64_t slots = 0;
#define DB_TRY(expr)                              \
  do {                                            \
    cudaError_t e__ = (expr);                     \
    if (e__ != cudaSuccess) {                     \
      st = cuda_status(e__, #expr);               \
      goto done;                                  \
    }                                             \
  } while (0)
  DB_TRY(cudaEventCreate(&e0));
  DB_TRY(cudaEventCreate(&e1));
  DB_TRY(cudaMalloc(&cnt, len * sizeof(uint64_t)));
  DB_TRY(cudaMalloc(&off, len * sizeof(uint64_t)));
  DB_TRY(cudaMalloc(&bsum, nb * sizeof(uint64_t)));
  DB_TRY(cudaEventRecord(e0, s));
  row_slots<<<(unsigned)((len + 255) / 256), 256, 0, s>>>(n, d_row, grp, noc, cnt);
  if ((st = check_launch("row_slots"))) goto done;
  scan_block<<<(unsigned)nb, ST, 0, s>>>(len, cnt, off, bsum);
  if ((st = check_launch("scan_block"))) goto done;
  scan_totals<<<1, ST, 0, s>>>(nb, bsum);
  if ((st = check_launch("scan_totals"))) goto done;
  add_block_offsets<<<(unsigned)((len + 255) / 256), 256, 0, s>>>(len, off, bsum);
  if ((st = check_launch("add_block_offsets"))) goto done;
  DB_TRY(cudaMemcpyAsync(&slots, off + n, sizeof slots, cudaMemcpyDeviceToHost, s));
  DB_TRY(cudaStreamSynchronize(s));
  {
    // every row's slot count is a multiple of th in NOC mode and th == 1 in COM mode
    const uint64_t columns = slots / th, tiles = (columns + thw - 1) / thw;
    const uint64_t lenAX = tiles * 2 * thw * th;
    const uint64_t lenSEC = (noc && th == 1) ? tiles : (noc ? tiles * thw : tiles * thw * th);
    if (lenAX > 0xFFFFFFFFull || lenSEC > 0xFFFFFFFFull) {
      st = ISPMV_ERR_OVERFLOW;
      goto done;
    }
    m->nrows = n;
    m->nnz = nnz;
    std::snprintf(m->mode, sizeof m->mode, "%s", mode);
    m->tileHW = thw;
    m->tileH = th;
    m->logTH = floor_log2_lt1024(th);
    m->lenCON = n;
    m->log = lg;
    m->tileN = (UIN)tiles;
    m->lenAX = (UIN)lenAX;
    m->lenSEC = (UIN)lenSEC;
    DB_TRY(cudaMalloc(&m->con, std::max<size_t>(1, n) * sizeof(UIN)));
    DB_TRY(cudaMalloc(&m->ax, std::max<uint64_t>(1, lenAX) * sizeof(FPT)));
    DB_TRY(cudaMalloc(&m->sec, std::max<uint64_t>(1, lenSEC) * sizeof(UIN)));
    DB_TRY(cudaMemsetAsync(m->ax, 0, lenAX * sizeof(FPT), s));
    DB_TRY(cudaMemsetAsync(m->sec, 0, lenSEC * sizeof(UIN), s));
    fill_axt<<<(unsigned)(((size_t)n * 32 + 255) / 256), 256, 0, s>>>(n, d_row, d_col, d_val, d_x, off, thw, th,
                                                                       noc, bs, lg, m->con, m->ax, m->sec);
    if ((st = check_launch("fill_axt"))) goto done;
    DB_TRY(cudaEventRecord(e1, s));
    DB_TRY(cudaEventSynchronize(e1));
    if (fd) {
      float ms = 0.f;
      DB_TRY(cudaEventElapsedTime(&ms, e0, e1));
      std::memset(fd, 0, sizeof *fd);
      if (noc && th == 1) std::snprintf(fd->name, sizeof fd->name, "AXT_NOC_H1_HW8");
      else if (noc) std::snprintf(fd->name, sizeof fd->name, "AXT_NOC_H%u_HW8", th);
      else std::snprintf(fd->name, sizeof fd->name, "AXT_COM_H1_HW8_BS%u", bs);
      fd->mfp = (double)m->lenAX * sizeof(FPT) + (double)m->lenSEC * sizeof(UIN);
      fd->beta = m->lenAX ? (double)nnz / (double)(m->lenAX >> 1) : 0.0;
      fd->ct = ms * 1e-3;
    }
  }
#undef DB_TRY
done:
  cudaFree(cnt);
  cudaFree(off);
  cudaFree(bsum);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st != ISPMV_OK) ispmv_dev_axt_free(m);
  return st;
}

// ---------------------------------------------------------------- K1 --
ISPMV_API int ispmv_dev_k1_free(str_matK1 *m) {
  if (!m) return ISPMV_ERR_ARG;
  cudaFree(m->permi);
  cudaFree(m->nmc);
  cudaFree(m->chp);
  cudaFree(m->val);
  cudaFree(m->col);
  std::memset(m, 0, sizeof *m);
  return ISPMV_OK;
}

// Copies a device-built K1's arrays into caller buffers (host or device;
// NULL skips one): permi (chunkNum+1)*8, nmc and chp chunkNum, val and col
// lenVC entries.  Synchronises `stream`.
ISPMV_API int ispmv_dev_k1_export(const str_matK1 *m, UIN *permi, UIN *nmc, UIN *chp, FPT *val, UIN *col,
                                  void *stream) {
  if (!m) return ISPMV_ERR_ARG;
  cudaStream_t s = as_stream(stream);
  const size_t cn = m->chunkNum;
  if (permi) ISPMV_TRY(cudaMemcpyAsync(permi, m->permi, (cn + 1) * 8 * sizeof(UIN), cudaMemcpyDefault, s));
  if (nmc && cn) ISPMV_TRY(cudaMemcpyAsync(nmc, m->nmc, cn * sizeof(UIN), cudaMemcpyDefault, s));
  if (chp && cn) ISPMV_TRY(cudaMemcpyAsync(chp, m->chp, cn * sizeof(UIN), cudaMemcpyDefault, s));
  if (val && m->lenVC) ISPMV_TRY(cudaMemcpyAsync(val, m->val, (size_t)m->lenVC * sizeof(FPT), cudaMemcpyDefault, s));
  if (col && m->lenVC) ISPMV_TRY(cudaMemcpyAsync(col, m->col, (size_t)m->lenVC * sizeof(UIN), cudaMemcpyDefault, s));
  ISPMV_TRY(cudaStreamSynchronize(s));
  return ISPMV_OK;
}

// getFormatDataK1 on the GPU from device CSR arrays; the struct's arrays
// come back as device pointers (ispmv_dev_k1_free); fd->ct is the GPU time.
ISPMV_API int ispmv_dev_build_k1(UIN n, UIN nnz, const UIN *d_row, const UIN *d_col, const FPT *d_val, str_matK1 *m,
                                 str_formatData *fd, void *stream) {
  if (!m || !d_row || n == 0 || (nnz && (!d_col || !d_val))) return ISPMV_ERR_ARG;
  cudaStream_t s = as_stream(stream);
  std::memset(m, 0, sizeof *m);
  const UIN cn = (n + 7) / 8;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  UIN *rl = nullptr, *rls = nullptr, *ids = nullptr;
  uint64_t *cnt = nullptr, *off = nullptr, *bsum = nullptr;
  void *tmp = nullptr;
  size_t tmp_bytes = 0;
  int st = ISPMV_OK;
  const size_t len = (size_t)cn + 1, nb = (len + SB - 1) / SB;
  uint64_t lenVC = 0;
#define DB_TRY(expr)                \
  do {                              \
    cudaError_t e__ = (expr);       \
    if (e__ != cudaSuccess) {       \
      st = cuda_status(e__, #expr); \
      goto done;                    \
    }                               \
  } while (0)
  DB_TRY(cudaEventCreate(&e0));
  DB_TRY(cudaEventCreate(&e1));
  DB_TRY(cudaMalloc(&rl, (size_t)n * sizeof(UIN)));
  DB_TRY(cudaMalloc(&rls, ((size_t)cn * 8) * sizeof(UIN)));
  DB_TRY(cudaMalloc(&ids, (size_t)n * sizeof(UIN)));
  DB_TRY(cudaMalloc(&m->permi, ((size_t)cn + 1) * 8 * sizeof(UIN)));
  DB_TRY(cudaMalloc(&m->nmc, std::max<size_t>(1, cn) * sizeof(UIN)));
  DB_TRY(cudaMalloc(&m->chp, std::max<size_t>(1, cn) * sizeof(UIN)));
  DB_TRY(cudaMalloc(&cnt, len * sizeof(uint64_t)));
  DB_TRY(cudaMalloc(&off, len * sizeof(uint64_t)));
  DB_TRY(cudaMalloc(&bsum, nb * sizeof(uint64_t)));
  DB_TRY(cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp_bytes, rl, rls, ids, m->permi, (int)n, 0,
                                                   32, s));
  DB_TRY(cudaMalloc(&tmp, std::max<size_t>(1, tmp_bytes)));
  DB_TRY(cudaEventRecord(e0, s));
  DB_TRY(cudaMemsetAsync(m->permi, 0, ((size_t)cn + 1) * 8 * sizeof(UIN), s));  // zero beyond n (M:851-852)
  DB_TRY(cudaMemsetAsync(rls, 0, (size_t)cn * 8 * sizeof(UIN), s));
  row_lengths<<<(unsigned)(((size_t)n + 255) / 256), 256, 0, s>>>(n, d_row, rl, ids);
  if ((st = check_launch("row_lengths"))) goto done;
  // stable: equal lengths keep ascending row ids
  DB_TRY(cub::DeviceRadixSort::SortPairsDescending(tmp, tmp_bytes, rl, rls, ids, m->permi, (int)n, 0, 32, s));
  chunk_widths<<<(unsigned)((len + 255) / 256), 256, 0, s>>>(cn, rls, m->nmc, cnt);
  if ((st = check_launch("chunk_widths"))) goto done;
  scan_block<<<(unsigned)nb, ST, 0, s>>>(len, cnt, off, bsum);
  if ((st = check_launch("scan_block"))) goto done;
  scan_totals<<<1, ST, 0, s>>>(nb, bsum);
  if ((st = check_launch("scan_totals"))) goto done;
  add_block_offsets<<<(unsigned)((len + 255) / 256), 256, 0, s>>>(len, off, bsum);
  if ((st = check_launch("add_block_offsets"))) goto done;
  DB_TRY(cudaMemcpyAsync(&lenVC, off + cn, sizeof lenVC, cudaMemcpyDeviceToHost, s));
  DB_TRY(cudaStreamSynchronize(s));
  if (lenVC > 0xFFFFFFFFull) {
    st = ISPMV_ERR_OVERFLOW;
    goto done;
  }
  m->nrows = n;
  m->nnz = nnz;
  m->chunkNum = cn;
  m->lenVC = (UIN)lenVC;
  DB_TRY(cudaMalloc(&m->val, std::max<uint64_t>(1, lenVC) * sizeof(FPT)));
  DB_TRY(cudaMalloc(&m->col, std::max<uint64_t>(1, lenVC) * sizeof(UIN)));
  DB_TRY(cudaMemsetAsync(m->val, 0, lenVC * sizeof(FPT), s));
  DB_TRY(cudaMemsetAsync(m->col, 0, lenVC * sizeof(UIN), s));
  fill_k1<<<(unsigned)(((size_t)n + 255) / 256), 256, 0, s>>>(n, d_row, d_col, d_val, m->permi, off, m->chp, m->val,
                                                               m->col);
  if ((st = check_launch("fill_k1"))) goto done;
  DB_TRY(cudaEventRecord(e1, s));
  DB_TRY(cudaEventSynchronize(e1));
  if (fd) {
    float ms = 0.f;
    DB_TRY(cudaEventElapsedTime(&ms, e0, e1));
    std::memset(fd, 0, sizeof *fd);
    std::snprintf(fd->name, sizeof fd->name, "K1");
    fd->mfp = 2.0 * cn * sizeof(UIN) + (double)m->lenVC * (sizeof(FPT) + sizeof(UIN)) + (double)n * sizeof(UIN) +
              (double)n * sizeof(FPT);
    fd->beta = m->lenVC ? (double)nnz / (double)m->lenVC : 0.0;
    fd->ct = ms * 1e-3;
  }
#undef DB_TRY
done:
  cudaFree(rl);
  cudaFree(rls);
  cudaFree(ids);
  cudaFree(cnt);
  cudaFree(off);
  cudaFree(bsum);
  cudaFree(tmp);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st != ISPMV_OK) ispmv_dev_k1_free(m);
  return st;
}
