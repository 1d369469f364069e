// plan_kernels.cuh - sm_100a SpMV kernels of the plan layer (fresh x per
// call, gathered through the read-only path / L2; values and columns are
// streamed once with evict-first loads).
//
// VT is the stored value type (double, or float for the reduced-byte form:
// FP32 multiply, FP64 accumulation).
#pragma once
#include "seg_engine.cuh"

namespace ispmv {
namespace pk {

constexpr int TPB = 256;

template <typename VT>
__device__ __forceinline__ double prod(VT v, double x);
template <>
__device__ __forceinline__ double prod<double>(double v, double x) { return v * x; }
template <>
__device__ __forceinline__ double prod<float>(float v, double x) { return (double)(v * __double2float_rn(x)); }

template <typename VT>
__device__ __forceinline__ double fmac(VT v, double x, double acc);
template <>
__device__ __forceinline__ double fmac<double>(double v, double x, double acc) { return fma(v, x, acc); }
template <>
__device__ __forceinline__ double fmac<float>(float v, double x, double acc) {
  return acc + (double)(v * __double2float_rn(x));
}

// ---------------------------------------------------------------- CSR --
// Vector CSR ("naive" CSR on the GPU): L lanes per row, shuffle reduction,
// overwrite / accumulate y.
template <typename VT, int L>
__global__ void __launch_bounds__(TPB) csr_vec(UIN n, const UIN *__restrict__ row, const UIN *__restrict__ col,
                                               const VT *__restrict__ val, const FPT *__restrict__ x,
                                               FPT *__restrict__ y, int beta) {
  const unsigned sub = threadIdx.x & (L - 1);
  const size_t r = ((size_t)blockIdx.x * TPB + threadIdx.x) / L;
  const bool live = r < n;
  double s = 0.0;
  if (live) {
    const UIN b = row[r], e = row[r + 1];
    for (UIN j = b + sub; j < e; j += L) s = fmac<VT>(ld_stream(val + j), ldg(x + ld_stream(col + j)), s);
  }
#pragma unroll
  for (int d = L / 2; d > 0; d >>= 1) s += __shfl_xor_sync(FULL, s, d);
  if (live && sub == 0) y[r] = beta ? s + y[r] : s;
}

// ---------------------------------------------------------------- AXC --
// 8 lanes per row, one 8-value brick per step (the reference's row loop,
// M:711-732, with x gathered from the column companion).
template <typename VT>
__global__ void __launch_bounds__(TPB) axc_rows(UIN n, const UIN *__restrict__ bptr, const UIN *__restrict__ col,
                                                const VT *__restrict__ val, const FPT *__restrict__ x,
                                                FPT *__restrict__ y, int beta) {
  const unsigned k = threadIdx.x & 7u;
  const size_t r = ((size_t)blockIdx.x * TPB + threadIdx.x) >> 3;
  const bool live = r < n;
  double s = 0.0;
  if (live) {
    const size_t b = (size_t)bptr[r] * 8, e = (size_t)bptr[r + 1] * 8;
    for (size_t p = b + k; p < e; p += 8) s = fmac<VT>(ld_stream(val + p), ldg(x + ld_stream(col + p)), s);
  }
  s += __shfl_xor_sync(FULL, s, 4);
  s += __shfl_xor_sync(FULL, s, 2);
  s += __shfl_xor_sync(FULL, s, 1);
  if (live && k == 0) y[r] = beta ? s + y[r] : s;
}

// ----------------------------------------------------------------- K1 --
// K1 orders rows by length (descending), so a chunk's rows are unrelated
// rows of the matrix and nearly every gather misses the lines its
// neighbours touched; the chunks' column counts nmc never increase.  The
// first `nlong` chunks (the long ones) get a warp each: 4 groups of 8 lanes
// (lane = row of the chunk) take every 4th column, 8 columns at a time, and
// combine their sums with two shuffles.  The rest go 4 chunks to a warp,
// 8 lanes each, also 8 columns at a time.  A lane keeps its 8 value/column
// loads and then its 8 gathers in flight together, with independent sums.
// SCATTER writes y[permi] (K1 with integrated reordering), else res in
// chunk order (then k1_order).  Every chunk column is one coalesced 64-byte
// load of values.
template <typename VT, int STRIDE>
__device__ __forceinline__ double k1_sum(const VT *__restrict__ val, const UIN *__restrict__ col,
                                         const FPT *__restrict__ x, size_t off, UIN k0, UIN m, unsigned lane8) {
  constexpr int U = 8;
  double acc[U];
#pragma unroll
  for (int u = 0; u < U; u++) acc[u] = 0.0;
  UIN k = k0;
  for (; k + (U - 1) * STRIDE < m; k += U * STRIDE) {
    const size_t p = off + (size_t)k * 8 + lane8;
    VT v[U];
    UIN cc[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      v[u] = ld_stream(val + p + (size_t)8 * STRIDE * u);
      cc[u] = ld_stream(col + p + (size_t)8 * STRIDE * u);
    }
    double xv[U];
#pragma unroll
    for (int u = 0; u < U; u++) xv[u] = ldg(x + cc[u]);
#pragma unroll
    for (int u = 0; u < U; u++) acc[u] = fmac<VT>(v[u], xv[u], acc[u]);
  }
#pragma unroll
  for (int u = 0; u < U; u++) {  // the last columns of this lane's share
    const UIN kk = k + (UIN)(u * STRIDE);
    if (kk < m) {
      const size_t p = off + (size_t)kk * 8 + lane8;
      acc[u] = fmac<VT>(ld_stream(val + p), ldg(x + ld_stream(col + p)), acc[u]);
    }
  }
  return ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
}

template <typename VT, bool SCATTER>
__global__ void __launch_bounds__(TPB) k1_chunks(UIN n, UIN chunkNum, UIN nlong, const UIN *__restrict__ chp,
                                                 const UIN *__restrict__ nmc, const UIN *__restrict__ permi,
                                                 const UIN *__restrict__ col, const VT *__restrict__ val,
                                                 const FPT *__restrict__ x, FPT *__restrict__ out, int beta) {
  pdl_trigger();
  const unsigned lane = threadIdx.x & 31u, lane8 = lane & 7u;
  const size_t w = ((size_t)blockIdx.x * TPB + threadIdx.x) >> 5;
  size_t c;
  double s;
  if (w < nlong) {  // one warp per long chunk: group g takes columns g, g + 4, ...
    c = w;
    s = k1_sum<VT, 4>(val, col, x, chp[c], lane >> 3, nmc[c], lane8);
    s += __shfl_xor_sync(FULL, s, 8);
    s += __shfl_xor_sync(FULL, s, 16);
    if (lane >= 8) return;
  } else {
    c = nlong + (w - nlong) * 4 + (lane >> 3);
    if (c >= chunkNum) return;
    s = k1_sum<VT, 1>(val, col, x, chp[c], 0, nmc[c], lane8);
  }
  const size_t i = c * 8 + lane8;
  if (SCATTER) {
    if (i < n) {
      const UIN r = permi[i];
      out[r] = beta ? s + out[r] : s;
    }
  } else {
    out[i] = s;
  }
}

// Warps of a K1 launch: one per long chunk, one per 4 other chunks.
inline size_t k1_warps(UIN chunkNum, UIN nlong) { return (size_t)nlong + ((size_t)(chunkNum - nlong) + 3) / 4; }

// K1's reorder (orderArrayK1): y in original row order from the chunk-order
// result; a programmatic dependent launch of k1_chunks where the stream
// allows it, so it first waits for that grid and its writes.
__global__ void k1_order(UIN n, const UIN *__restrict__ permi, const FPT *__restrict__ res, FPT *__restrict__ y,
                         int beta) {
  pdl_wait();
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const UIN r = permi[i];
    y[r] = beta ? res[i] + y[r] : res[i];
  }
}

// ------------------------------------------------------- AXT NOC, th>1 --
// Unit = tile column of th slots (row id: sec[8*T + c]).  th % 4 == 0: each
// step the warp loads 4 consecutive sub-rows of a tile (32 consecutive
// slots), adds them per column, and after th/4 steps reduces the 4 partials
// of each column with 2 shuffles; 4 tiles make a batch of 32 columns.
template <typename VT>
__global__ void __launch_bounds__(TPB) noc_hn(size_t nunits, size_t nseg, UIN th, UIN useg, const UIN *__restrict__ urow,
                                              const UIN *__restrict__ col, const VT *__restrict__ val,
                                              const FPT *__restrict__ x, seg::Out o) {
  pdl_trigger();
  const unsigned lane = threadIdx.x & 31u;
  const size_t segid = ((size_t)blockIdx.x * TPB + threadIdx.x) >> 5;
  if (segid >= nseg) return;
  const size_t u0 = segid * useg;  // useg is a multiple of 32 (4 tiles)
  const size_t u1 = min(u0 + useg, nunits);
  seg::State st{NO_ROW, 0.0, false};
  const size_t tslots = (size_t)th * 8;
  for (size_t ub = u0; ub < u1; ub += 32) {
    double mine = 0.0;
    for (int tt = 0; tt < 4; tt++) {
      const size_t T = ub / 8 + tt;
      double p = 0.0;
      if (T * 8 < u1) {
        const size_t base = T * tslots + lane;
        if (th % 4 == 0) {
          for (UIN R = 0; R < th; R += 4) {
            const size_t q = base + (size_t)R * 8;
            p = fmac<VT>(ld_stream(val + q), ldg(x + ld_stream(col + q)), p);
          }
        } else {
          // generic tileH: lane = (group g = lane/8, column c): sub-rows g, g+4, ...
          for (UIN R = lane >> 3; R < th; R += 4) {
            const size_t q = T * tslots + (size_t)R * 8 + (lane & 7u);
            p = fmac<VT>(ld_stream(val + q), ldg(x + ld_stream(col + q)), p);
          }
        }
      }
      p += __shfl_xor_sync(FULL, p, 8);
      p += __shfl_xor_sync(FULL, p, 16);
      if ((lane >> 3) == (unsigned)tt) mine = p;
    }
    const size_t u = ub + lane;
    const bool live = u < u1;
    const UIN r = live ? urow[u] : NO_ROW;
    seg::batch(mine, r, live, st, o, segid);
  }
  seg::finish(st, o, segid);
}

}  // namespace pk
}  // namespace ispmv
