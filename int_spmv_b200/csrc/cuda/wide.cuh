// wide.cuh - the slot-stream SpMV over a lane-interleaved copy of the
// stream, 8 or 16 slots per lane, with the x bands a CTA's rows need staged
// in shared memory.
//
// Why: on B200 the 4-slot-per-lane kernel (stream_ldg) is bound by the L1
// data path, not by HBM.  A warp-wide gather of 32 unrelated columns costs
// one L1 wavefront per distinct 128-byte line (about one per nonzero), and
// its segmented warp scan runs once per 128 slots (about 1.7 instructions
// per nonzero).  This kernel:
//   - runs one warp scan per 32*SPL slots (SPL = 16: 512), so the
//     warp-level reduction costs about 0.15 instructions per nonzero;
//   - reads values and columns with coalesced 16-byte loads from a copy of
//     the stream stored lane-interleaved: per batch of 32*SPL slots, lane l
//     owns the SPL consecutive slots b + SPL*l + k, and element (l, k) sits at
//     b + (k / V)*32*V + l*V + k % V with V = 16 / sizeof(element), so every
//     vector load of the warp is 512 contiguous bytes;
//   - gathers x through L1/L2 with plain loads; variants gather a column
//     that falls in the CTA's x window from shared memory, or every column
//     through the texture pipe.  Which path serves a column does not change
//     the result;
//   - FP32-value plans gather an FP32 copy of x made once per product, and
//     columns may be 16-bit deltas to a per-batch base (D16).
// The row reduction is the slot stream's: rows are contiguous runs of
// slots, row starts are bits of `heads` (slot order), a warp owns a segment
// of slots and leaves two (row, partial) records per segment for
// seg::fixup.  A row is written by the lane that ends it.  Every row is
// written exactly once, without atomics, and the summation order is fixed,
// so results are bitwise repeatable.
//
// stream_wide_tma is the same reduction fed by 1D bulk copies
// (cp.async.bulk, no multicast) into a per-warp ring of stages in shared
// memory: one lane keeps the next stages of its warp's segments in flight,
// so the value/column stream leaves both the warp's critical path and the
// L1 load pipe.
#pragma once
#include "sss.cuh"

namespace ispmv {
namespace wide {

// Position of slot s in the lane-interleaved copy (32*spl-slot batches,
// v elements per vector load).
__host__ __device__ inline size_t il_pos(size_t s, unsigned spl, unsigned v) {
  const size_t bt = 32u * spl;
  const size_t b = s / bt * bt;
  const unsigned r = (unsigned)(s - b), l = r / spl, k = r % spl;
  return b + (size_t)(k / v) * 32u * v + (size_t)l * v + k % v;
}

// il_pos with the slots per lane (0: slot order, 8 or 16) and the elements
// per vector load known at compile time: shifts and masks, no division.
template <int SPL, unsigned V>
__device__ __forceinline__ size_t il_pos_c(size_t s) {
  if constexpr (SPL == 0) {
    return s;
  } else {
    static_assert((SPL & (SPL - 1)) == 0 && (V & (V - 1)) == 0, "powers of two");
    constexpr size_t BT = 32u * SPL;
    const unsigned r = (unsigned)(s & (BT - 1)), l = r / SPL, k = r % SPL;
    return (s & ~(BT - 1)) + (size_t)(k / V) * 32u * V + (size_t)l * V + k % V;
  }
}

template <typename VT, int SPL>
struct Vals;
template <int SPL>
struct Vals<double, SPL> {
  double2 q[SPL / 2];
  __device__ __forceinline__ void get(const double *v, size_t b, unsigned lane) {
#pragma unroll
    for (int i = 0; i < SPL / 2; i++) q[i] = ld_stream(reinterpret_cast<const double2 *>(v + b + 64 * i + 2 * lane));
  }
  __device__ __forceinline__ double operator[](int k) const { return (k & 1) ? q[k >> 1].y : q[k >> 1].x; }
};
template <int SPL>
struct Vals<float, SPL> {
  float4 q[SPL / 4];
  __device__ __forceinline__ void get(const float *v, size_t b, unsigned lane) {
#pragma unroll
    for (int i = 0; i < SPL / 4; i++) q[i] = ld_stream(reinterpret_cast<const float4 *>(v + b + 128 * i + 4 * lane));
  }
  __device__ __forceinline__ float operator[](int k) const {
    const float4 &t = q[k >> 2];
    return (k & 3) == 0 ? t.x : (k & 3) == 1 ? t.y : (k & 3) == 2 ? t.z : t.w;
  }
};

template <int SPL>
struct Cols {
  uint4 q[SPL / 4];
  __device__ __forceinline__ void get(const UIN *c, size_t b, unsigned lane) {
#pragma unroll
    for (int i = 0; i < SPL / 4; i++) q[i] = ld_stream(reinterpret_cast<const uint4 *>(c + b + 128 * i + 4 * lane));
  }
  __device__ __forceinline__ UIN operator[](int k) const {
    const uint4 &t = q[k >> 2];
    return (k & 3) == 0 ? t.x : (k & 3) == 1 ? t.y : (k & 3) == 2 ? t.z : t.w;
  }
};

// SPL 16-bit column deltas of one lane (lane-interleaved, 8 per 16-byte load).
template <int SPL>
struct Deltas {
  uint4 q[SPL / 8];
  __device__ __forceinline__ void get(const uint16_t *d, size_t b, unsigned lane) {
#pragma unroll
    for (int i = 0; i < SPL / 8; i++) q[i] = ld_stream(reinterpret_cast<const uint4 *>(d + b + 256 * i + 8 * lane));
  }
  __device__ __forceinline__ UIN operator[](int k) const {
    const uint4 &t = q[k >> 3];
    const int w = (k & 7) >> 1;
    const UIN word = w == 0 ? t.x : w == 1 ? t.y : w == 2 ? t.z : t.w;
    return (k & 1) ? word >> 16 : word & 0xFFFFu;
  }
};

// acc + v*x in the plan's value form: FP64 values fused multiply-add; FP32
// values multiplied in FP32 (x rounded to FP32, or gathered from the plan's
// FP32 copy of x, the same value) and added in FP64.
__device__ __forceinline__ double madd(double v, double x, double acc) { return fma(v, x, acc); }
__device__ __forceinline__ double madd(float v, double x, double acc) {
  return acc + (double)(v * __double2float_rn(x));
}
__device__ __forceinline__ double madd(float v, float x, double acc) { return acc + (double)(v * x); }

// x rounded to FP32 once per product, for FP32-value plans: their gathers
// then move 4 bytes per slot and an L1 line serves 32 columns.  VEC: x and
// x32 are 16- and 8-byte aligned, two elements per thread and step.
template <bool VEC>
__global__ void __launch_bounds__(256) x_to_f32(size_t n, const FPT *__restrict__ x, float *__restrict__ x32) {
  pdl_trigger();  // the product's main kernel may start loading its stream now
  const size_t stride = (size_t)gridDim.x * 256;
  size_t i = (size_t)blockIdx.x * 256 + threadIdx.x;
  if constexpr (VEC) {
    const size_t n2 = n / 2;
    for (; i < n2; i += stride) {
      const double2 v = __ldcs(reinterpret_cast<const double2 *>(x) + i);
      reinterpret_cast<float2 *>(x32)[i] = make_float2(__double2float_rn(v.x), __double2float_rn(v.y));
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && (n & 1)) x32[n - 1] = __double2float_rn(x[n - 1]);
  } else {
    for (; i < n; i += stride) x32[i] = __double2float_rn(__ldg(x + i));
  }
}

// The x window a CTA stages (NW = 1): columns [lo, lo + len) at shared-memory
// offset lo + delta (u32 arithmetic, modulo 2^32).
template <int NW>
struct Bands {
  UIN lo[NW > 0 ? NW : 1], len[NW > 0 ? NW : 1], delta[NW > 0 ? NW : 1];
};

// x[c]: from the shared-memory window when c falls in it, else through
// L1/L2.  Two predicated loads into one register: the shared-memory load
// runs on the lanes whose column is in the window, the global load on the
// others.
template <int NW>
__device__ __forceinline__ double gather(const Bands<NW> &w, uint32_t sx_addr, const FPT *__restrict__ x, UIN c) {
  if constexpr (NW == 0) {
    return __ldg(x + c);
  } else {
    uint32_t in = 0, off = 0;
#pragma unroll
    for (int k = 0; k < NW; k++) {
      if (c - w.lo[k] < w.len[k]) {  // window starts lie in [0, n]: the unsigned difference is exact
        in = 1;
        off = c + w.delta[k];
      }
    }
    double v;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "setp.ne.u32 p, %3, 0;\n"
        "@p ld.shared.f64 %0, [%1];\n"
        "@!p ld.global.nc.f64 %0, [%2];\n"
        "}\n"
        : "=d"(v)
        : "r"(sx_addr + 8u * off), "l"(x + c), "r"(in));
    return v;
  }
}

// One batch of 32*SPL slots: lane l holds the values v[k] and gathered x
// values xv[k] of slots b + SPL*l + k, and `bits`, its SPL row-start bits
// (bit k = slot k).  Each lane sums its slots in slot order into `pre`
// (slots before its first row start), the rows that start and end in it,
// and `acc` (the run from its last row start); one segmented warp scan then
// joins the pieces of rows that cross lanes.  When no lane of the warp
// holds two row starts (rows longer than SPL slots), the lane pass is two
// predicated multiply-adds per slot; otherwise the rows that end inside a
// lane are written as they end.  Both paths add the same products in the
// same order, so the result does not depend on the path.  Every row goes to
// y (or to the segment's head record) from the lane that ends it.
template <typename VT, typename XT, int SPL>
__device__ __forceinline__ void batch(const VT (&v)[SPL], const XT (&xv)[SPL], unsigned bits, sss::Run &st,
                                      const seg::Out &o) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned cnt = __popc(bits);
  // row starts before my slots (ex) and in the batch (tot): counts summed
  // bit plane by bit plane with ballots, keeping the shuffle (LSU) pipe free
  constexpr int PLANES = SPL >= 16 ? 5 : SPL >= 8 ? 4 : 3;
  const unsigned lt = sss::lanemask_le() >> 1;  // lanes below mine
  unsigned ex = 0, tot = 0;
#pragma unroll
  for (int q = 0; q < PLANES; q++) {
    const unsigned m = __ballot_sync(FULL, (cnt >> q) & 1u);
    ex += (unsigned)__popc(m & lt) << q;
    tot += (unsigned)__popc(m) << q;
  }
  // ex = entry of the row open at my first slot
  const UIN rb = st.rbase + ex;     // row of my first start
  const int first = cnt ? __ffs(bits) - 1 : SPL;
  double pre = 0.0, acc = 0.0;
  if (__all_sync(FULL, cnt <= 1u)) {
#pragma unroll
    for (int k = 0; k < SPL; k++) {
      if (k < first) pre = madd(v[k], xv[k], pre);
      else acc = madd(v[k], xv[k], acc);
    }
  } else {
    UIN r = rb;  // row of the run being summed, once past my first start
#pragma unroll
    for (int k = 0; k < SPL; k++) {
      if ((bits >> k) & 1u) {
        if (k > first) {  // a row that starts and ends in this lane
          seg::write_row(o, r, acc);  // never the segment's open row: it started in this segment
          r++;
        } else {
          pre = acc;
        }
        acc = 0.0;
      }
      acc = madd(v[k], xv[k], acc);
    }
    if (!cnt) {
      pre = acc;
      acc = 0.0;
    }
  }
  if (lane == 0 && st.carry) pre += st.csum;
  // lanes' leading and trailing pieces: one segmented warp scan whose
  // windows stop at the lane holding the row's start
  const bool f = cnt != 0;
  const unsigned F = __ballot_sync(FULL, f) & sss::lanemask_le();
  const int start = F ? 31 - __clz(F) : 0;
  const int reach = (int)lane - start;
  double I = f ? acc : pre;
  // only as many steps as the longest window needs (rows spanning few
  // lanes: one or two); a step whose distance exceeds every lane's reach
  // adds nothing, so the sums are the same bits as with all five steps
  const int maxreach = (int)__reduce_max_sync(FULL, (unsigned)reach);
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    if (d > maxreach) break;
    const double u = __shfl_up_sync(FULL, I, d);
    if (reach >= d) I += u;
  }
  double E = __shfl_up_sync(FULL, I, 1);
  if (lane == 0) E = 0.0;
  // the run open at my lane's start ends at my first row start
  if (f && (lane > 0 || !(bits & 1u) || st.carry)) sss::emit(o, st, rb - 1u, E + pre);
  st.csum = __shfl_sync(FULL, I, 31);
  st.carry = true;
  st.rbase += tot;
}

// Plain-load form.  MINB CTAs of WARPS*32 threads per SM bound the
// registers.  NW = 1 with STG (the CTA's x window in shared memory), else 0
// (every gather through L1/L2).
// D16: columns as 16-bit deltas to a per-batch base column (nw.cmeta, one
// per batch of 32*SPL slots), lane-interleaved like the values; a batch whose
// columns span more than 16 bits keeps its u32 columns in nw.esc (cmeta =
// ESCAPE | its index there).
// TEX: x is gathered with texture fetches (tex1Dfetch on `xtex`, a linear
// texture over x) instead of global loads: the texture pipe of L1TEX serves
// the gathers while the load/store pipe streams values and columns.
// STG: one window per CTA chosen by the plan (xw.tlo/xw.tlen: the densest
// interval of the CTA's columns), copied into shared memory by one bulk copy
// (cp.async.bulk, no multicast) on an mbarrier; x must be 16-byte aligned
// (the host checks).  The copy leaves the L1 load pipe to the gathers and
// costs no load loop.  Each warp waits for it (bounded) only before its
// first gathers, after its first batch's values and columns are on their
// way, so the copy's latency overlaps the stream's (2% faster on the
// power-law matrix than a wait at CTA start).
// LO (FP32 values, FP64 x): in segments whose rows need it, a BF16 residual
// per slot (nw.lo16 at nw.lo_off[segment], lane-interleaved like D16's
// deltas); such a segment multiplies hi + lo (exact in FP64 unless lo is
// below 2^-45 of hi) by x in FP64, the others multiply in FP32.
// PFC: the next batch's columns are loaded one batch ahead (u32 columns),
// so a batch's gathers issue without waiting for its column load.
template <typename VT, typename XT, int SPL, int NW, int WARPS, int MINB, bool D16 = false, bool TEX = false,
          bool STG = false, bool LO = false, bool PFC = false>
__global__ void __launch_bounds__(WARPS * 32, MINB)
    stream_wide(size_t nslots, size_t nslots_pad, size_t seg_slots, size_t nseg, const VT *__restrict__ val,
                const UIN *__restrict__ col, const UIN *__restrict__ heads, const UIN *__restrict__ segh,
                sss::XWin xw, const XT *__restrict__ x, seg::Out o, sss::Narrow nw = {},
                cudaTextureObject_t xtex = 0) {
  static_assert(NW == (STG ? 1 : 0), "the shared-memory window is the staged form's");
  static_assert(!STG || sizeof(XT) == 8, "the window holds FP64 x");
  static_assert(!LO || (sizeof(VT) == 4 && sizeof(XT) == 8), "lo-words correct FP32 values against FP64 x");
  static_assert(!(PFC && D16), "column prefetch reads u32 columns");
  constexpr int BT = 32 * SPL;
  constexpr unsigned MASK = SPL == 32 ? 0xffffffffu : (1u << SPL) - 1u;
  extern __shared__ __align__(16) double sx[];
  pdl_trigger();  // the row fix-up may launch now; it waits for this grid before it reads
  const unsigned lane = threadIdx.x & 31u;
  const size_t seg0 = (size_t)blockIdx.x * WARPS;
  const size_t segid = seg0 + (threadIdx.x >> 5);
  Bands<NW> w{};
  __shared__ uint64_t wbar;
  UIN wlen = 0;  // STG: the window's length, 0 once this warp has seen it land
  if constexpr (STG) {
    const UIN lo = __ldg(xw.tlo + blockIdx.x), len = __ldg(xw.tlen + blockIdx.x);
    if (threadIdx.x == 0 && len) {
      tma::bar_init(&wbar, 1);
      tma::fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && len) {
      tma::bar_expect_tx(&wbar, len * 8u);
      tma::bulk_g2s(sx, x + lo, len * 8u, &wbar);
    }
    // each warp waits for the window just before its first gathers, so that
    // its first batch's values and columns load during the copy.  Warp 0
    // (thread 0, the copy's issuer) always owns a segment, so the CTA, and
    // its shared memory, outlives the copy.
    wlen = len;
    w.lo[0] = lo;
    w.len[0] = len;
    w.delta[0] = 0u - lo;
  }
  if (segid >= nseg) return;
  const uint32_t sxa = tma::smem_addr(sx);
  const size_t s0 = segid * seg_slots;
  const size_t s1 = min(s0 + seg_slots, nslots_pad);
  const int nbat = (int)((s1 - s0) / BT);
  sss::Run st;
  sss::begin(st, o, segid, segh[segid], __ldg(heads + (s0 >> 5)));
  UIN lo_base = NO_ROW;
  if constexpr (LO) lo_base = __ldg(nw.lo_off + segid);
  Cols<SPL> cnext;  // PFC: the columns of batch j + 1
  if constexpr (PFC) {
    if (nbat > 0) cnext.get(col, s0, lane);
  }
  for (int j = 0; j < nbat; j++) {
    const size_t b = s0 + (size_t)j * BT;
    Vals<VT, SPL> v;
    v.get(val, b, lane);
    UIN c[SPL];
    if constexpr (D16) {
      const UIN m = __ldg(nw.cmeta + b / BT);  // the same word for the whole warp
      if (m & sss::ESCAPE) {
        Cols<SPL> e;
        e.get(nw.esc + (size_t)(m & ~sss::ESCAPE) * BT, 0, lane);
#pragma unroll
        for (int k = 0; k < SPL; k++) c[k] = e[k];
      } else {
        Deltas<SPL> d;
        d.get(nw.col16, b, lane);
#pragma unroll
        for (int k = 0; k < SPL; k++) c[k] = m + d[k];
      }
    } else if constexpr (PFC) {
#pragma unroll
      for (int k = 0; k < SPL; k++) c[k] = cnext[k];
      if (j + 1 < nbat) cnext.get(col, b + BT, lane);
    } else {
      Cols<SPL> e;
      e.get(col, b, lane);
#pragma unroll
      for (int k = 0; k < SPL; k++) c[k] = e[k];
    }
    const unsigned bits = (__ldg(heads + (b >> 5) + ((SPL * lane) >> 5)) >> ((SPL * lane) & 31u)) & MASK;
    if constexpr (sizeof(XT) == 4) {
      // FP32 x is written by x_to_f32, of which this kernel is a programmatic
      // dependent: its first batch's values and columns are loaded, now wait
      // for that grid and its writes before the first gather
      if (j == 0) pdl_wait();
    }
    if constexpr (STG) {
      if (wlen) {  // first batch: the window must have landed (bounded wait)
        wlen = 0;
        if (!__all_sync(FULL, tma::bar_wait(&wbar, 0))) {
          if (lane == 0) {
            if (xw.status) atomicCAS(xw.status, 0, ISPMV_ERR_TIMEOUT);
            (void)tma::bar_wait(&wbar, 0);  // the copy in flight, before the CTA's shared memory goes
          }
          return;
        }
      }
    }
    XT xv[SPL];
#pragma unroll
    for (int k = 0; k < SPL; k++) {
      if constexpr (NW > 0) {
        xv[k] = gather<NW>(w, sxa, x, c[k]);
      } else if constexpr (TEX) {
        if constexpr (sizeof(XT) == 8) {
          const int2 t = tex1Dfetch<int2>(xtex, (int)c[k]);
          xv[k] = __hiloint2double(t.y, t.x);
        } else {
          xv[k] = tex1Dfetch<float>(xtex, (int)c[k]);
        }
      } else {
        xv[k] = __ldg(x + c[k]);
      }
    }
    VT vv[SPL];
#pragma unroll
    for (int k = 0; k < SPL; k++) vv[k] = v[k];
    const size_t sl = b + (size_t)SPL * lane;
    if (sl + SPL > nslots) {  // the stream's zero padding adds nothing, whatever x holds
#pragma unroll
      for (int k = 0; k < SPL; k++)
        if (sl + k >= nslots) xv[k] = (XT)0;
    }
    if constexpr (LO) {
      if (lo_base != NO_ROW) {  // the segment's residuals: FP64 values hi + lo
        Deltas<SPL> lw;
        lw.get(nw.lo16 + lo_base, b - s0, lane);
        double vd[SPL];
#pragma unroll
        for (int k = 0; k < SPL; k++) vd[k] = (double)vv[k] + sss::bf16_to_double((uint16_t)lw[k]);
        batch<double, XT, SPL>(vd, xv, bits, st, o);
        continue;
      }
    }
    batch<VT, XT, SPL>(vv, xv, bits, st, o);
  }
  sss::finish(st, o);
}

// Bytes of one stage (one batch of 32*SPL slots: values, columns, bitmap)
// and of the dynamic shared memory of stream_wide_tma.
template <typename VT, int SPL>
constexpr uint32_t stage_bytes() {
  return 32u * SPL * (uint32_t)sizeof(VT) + 32u * SPL * 4u + 4u * SPL;
}
template <typename VT, int SPL, int STAGES, int WARPS>
constexpr size_t tma_smem_bytes() {
  return ((WARPS * STAGES * 8 + 127) / 128) * 128 + (size_t)WARPS * STAGES * stage_bytes<VT, SPL>();
}

// Staged form: persistent warps; warp g of G takes segments g, g + G, ...
// Lane 0 keeps the warp's next STAGES batches in flight as three bulk
// copies each (values, columns, bitmap words) completing on the stage's
// mbarrier.  Waits are bounded: a wait that gives up records
// ISPMV_ERR_TIMEOUT in *status, the warp stops, and lane 0 waits (bounded)
// for its copies still in flight before the CTA exits.
template <typename VT, int SPL, int STAGES, int WARPS>
__global__ void __launch_bounds__(WARPS * 32)
    stream_wide_tma(size_t nslots, size_t nslots_pad, size_t seg_slots, size_t nseg, const VT *__restrict__ val,
                    const UIN *__restrict__ col, const UIN *__restrict__ heads, const UIN *__restrict__ segh,
                    const FPT *__restrict__ x, seg::Out o, int *status) {
  pdl_trigger();
  constexpr int BT = 32 * SPL;
  constexpr unsigned MASK = SPL == 32 ? 0xffffffffu : (1u << SPL) - 1u;
  constexpr uint32_t VB = BT * sizeof(VT), CB = BT * 4, HB = BT / 8, STB = stage_bytes<VT, SPL>();
  static_assert(VB % 16 == 0 && CB % 16 == 0 && HB % 16 == 0, "bulk copies move multiples of 16 bytes");
  extern __shared__ __align__(128) unsigned char smem[];
  const int wib = threadIdx.x >> 5;
  const unsigned lane = threadIdx.x & 31u;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem) + wib * STAGES;
  unsigned char *ring = smem + ((WARPS * STAGES * 8 + 127) / 128) * 128 + (size_t)wib * STAGES * STB;
  const size_t gw = (size_t)blockIdx.x * WARPS + wib, GW = (size_t)gridDim.x * WARPS;
  if (gw >= nseg) return;
  if (lane == 0) {
    for (int s = 0; s < STAGES; s++) tma::bar_init(&bars[s], 1);
    tma::fence_barrier_init();
  }
  __syncwarp();
  const uint64_t pol = tma::policy_evict_first();
  // producer position (lane 0): segment and batch of the next copy
  size_t pseg = gw;
  uint32_t pbat = 0;
  auto issue = [&](int s) {
    const size_t b = pseg * seg_slots + (size_t)pbat * BT;
    unsigned char *dst = ring + (size_t)s * STB;
    tma::bar_expect_tx(&bars[s], VB + CB + HB);
    tma::bulk_g2s(dst, val + b, VB, &bars[s], pol);
    tma::bulk_g2s(dst + VB, col + b, CB, &bars[s], pol);
    tma::bulk_g2s(dst + VB + CB, heads + b / 32, HB, &bars[s], pol);
    if (++pbat >= sss::seg_nst<BT>(pseg, seg_slots, nslots_pad)) {
      pseg += GW;
      pbat = 0;
    }
  };
  int inflight = 0;  // copies issued and not yet consumed (lane 0's count)
  if (lane == 0)
    for (int s = 0; s < STAGES && pseg < nseg; s++) {
      issue(s);
      inflight++;
    }
  size_t cseg = gw;
  uint32_t cbat = 0, t = 0;
  sss::Run st;
  bool gaveup = false;
  while (cseg < nseg) {
    const int s = (int)(t % STAGES);
    // the lanes poll independently; they stop together if any gave up
    if (!__all_sync(FULL, tma::bar_wait(&bars[s], (t / STAGES) & 1u))) {
      if (lane == 0 && status) atomicCAS(status, 0, ISPMV_ERR_TIMEOUT);
      gaveup = true;
      break;
    }
    const unsigned char *stage = ring + (size_t)s * STB;
    const size_t b = cseg * seg_slots + (size_t)cbat * BT;
    const UIN *shd = reinterpret_cast<const UIN *>(stage + VB + CB);
    if (cbat == 0) sss::begin(st, o, cseg, segh[cseg], shd[0]);
    const unsigned bits = (shd[(SPL * lane) >> 5] >> ((SPL * lane) & 31u)) & MASK;
    UIN c[SPL];
#pragma unroll
    for (int i = 0; i < SPL / 4; i++) {
      const uint4 q = *reinterpret_cast<const uint4 *>(stage + VB + 16u * (32u * i + lane));
      c[4 * i] = q.x;
      c[4 * i + 1] = q.y;
      c[4 * i + 2] = q.z;
      c[4 * i + 3] = q.w;
    }
    double xv[SPL];
#pragma unroll
    for (int k = 0; k < SPL; k++) xv[k] = __ldg(x + c[k]);
    VT v[SPL];
    if constexpr (sizeof(VT) == 8) {
#pragma unroll
      for (int i = 0; i < SPL / 2; i++) {
        const double2 q = *reinterpret_cast<const double2 *>(stage + 16u * (32u * i + lane));
        v[2 * i] = q.x;
        v[2 * i + 1] = q.y;
      }
    } else {
#pragma unroll
      for (int i = 0; i < SPL / 4; i++) {
        const float4 q = *reinterpret_cast<const float4 *>(stage + 16u * (32u * i + lane));
        v[4 * i] = q.x;
        v[4 * i + 1] = q.y;
        v[4 * i + 2] = q.z;
        v[4 * i + 3] = q.w;
      }
    }
    // every lane has read the stage: refill it with the batch STAGES ahead
    __syncwarp();
    if (lane == 0) {
      inflight--;
      if (pseg < nseg) {
        tma::fence_proxy_async();
        issue(s);
        inflight++;
      }
    }
    const size_t sl = b + (size_t)SPL * lane;
    if (sl + SPL > nslots) {  // the stream's zero padding adds nothing, whatever x holds
#pragma unroll
      for (int k = 0; k < SPL; k++)
        if (sl + k >= nslots) xv[k] = 0.0;
    }
    batch<VT, double, SPL>(v, xv, bits, st, o);
    if (++cbat >= sss::seg_nst<BT>(cseg, seg_slots, nslots_pad)) {
      sss::finish(st, o);
      cseg += GW;
      cbat = 0;
    }
    t++;
  }
  if (gaveup && lane == 0) {
    // the copies still in flight complete on the next phases of their stages
    for (int i = 0; i < inflight; i++) {
      const uint32_t tt = t + (uint32_t)i;
      (void)tma::bar_wait(&bars[tt % STAGES], (tt / STAGES) & 1u);
    }
  }
}

}  // namespace wide
}  // namespace ispmv
