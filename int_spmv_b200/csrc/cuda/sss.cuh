// sss.cuh - the segmented slot stream kernel: y = A x over a stream of
// (value, column) slots in which every row's slots are contiguous and row
// starts are marked in a bitmap (bit s of `heads` = a non-empty row starts
// at slot s).  The compacted AXT layout (CSR order), the AXT tileH=1 tile
// stream and the AXC brick stream are all such streams (the latter two with
// zero padding inside each row's last tile / brick).
//
// A warp owns a segment of slots and walks it in batches of 128: lane l
// takes the 4 consecutive slots 4l..4l+3.  Runs that start and end inside a
// lane go straight to y; each lane's leading piece (before its first row
// start) and trailing piece (from its last row start) are combined across
// lanes by one segmented warp scan whose windows are clamped at the row
// start (no flag shuffles).  The run open at the segment's first slot and
// the one open at its end become the segment's two records (seg::fixup adds
// records of the same row and writes y).  Rows are compressed indices (the
// count of row starts before a slot); `rowmap` maps them to real rows when
// some rows are empty.
#pragma once
#include "plan_kernels.cuh"
#include "tma.cuh"

namespace ispmv {
namespace sss {

constexpr int BATCH = 128;  // slots per batch of the staged kernel (4 per lane)

struct Run {
  UIN rbase;   // row starts before the current batch
  UIN row_a;   // the run open at the segment's first slot (NO_ROW if it starts there)
  double csum; // partial of the run open at the current batch start
  bool carry;  // that run has slots in this segment
  UIN seg;
};

__device__ __forceinline__ void emit(const seg::Out &o, const Run &st, UIN row, double v) {
  if (row == st.row_a) {
    o.rec_row[2 * (size_t)st.seg] = row;
    o.rec_sum[2 * (size_t)st.seg] = v;
  } else {
    seg::write_row(o, row, v);
  }
}

__device__ __forceinline__ void begin(Run &st, const seg::Out &o, size_t segid, UIN rbase, UIN first_word) {
  st.seg = (UIN)segid;
  st.rbase = rbase;
  st.carry = false;
  st.csum = 0.0;
  st.row_a = (first_word & 1u) ? NO_ROW : rbase - 1u;
  if ((threadIdx.x & 31u) == 0) {
    o.rec_row[2 * segid] = NO_ROW;
    o.rec_sum[2 * segid] = 0.0;
  }
}

// Bitmap words of one batch of 32*SPL slots.
template <int SPL>
struct Words;
template <>
struct Words<2> {
  uint2 w;
  __device__ __forceinline__ UIN get(int i) const { return i == 0 ? w.x : w.y; }
};
template <>
struct Words<4> {
  uint4 w;
  __device__ __forceinline__ UIN get(int i) const { return i == 0 ? w.x : i == 1 ? w.y : i == 2 ? w.z : w.w; }
};

// One batch of 32*SPL slots; lane l holds slots SPL*l .. SPL*l+SPL-1 with
// products p, the batch's bitmap words hw.
template <int SPL>
__device__ __forceinline__ void batch(const double (&p)[SPL], const Words<SPL> &hw, Run &st, const seg::Out &o) {
  constexpr unsigned LPW = 32 / SPL;  // lanes per bitmap word
  const unsigned lane = threadIdx.x & 31u;
  const unsigned q = lane / LPW, sh = SPL * (lane % LPW);
  unsigned cnt[SPL], before = 0, tot = 0;
#pragma unroll
  for (int i = 0; i < SPL; i++) {
    cnt[i] = __popc(hw.get(i));
    before += (i < (int)q) ? cnt[i] : 0u;
    tot += cnt[i];
  }
  UIN myw = hw.get(0);
#pragma unroll
  for (int i = 1; i < SPL; i++)
    if ((int)q == i) myw = hw.get(i);
  const unsigned bits = (myw >> sh) & ((1u << SPL) - 1u);
  const UIN rb = st.rbase + before + __popc(myw & ((1u << sh) - 1u));  // row of my first start
  double pre = (lane == 0 && st.carry) ? st.csum : 0.0, run = 0.0;
  if (bits == 0) {
    double a = 0.0;
#pragma unroll
    for (int k = 0; k < SPL; k++) a += p[k];
    pre += a;
  } else {
    unsigned nh = 0;
#pragma unroll
    for (int k = 0; k < SPL; k++) {
      if ((bits >> k) & 1u) {
        if (nh) emit(o, st, rb + nh - 1u, run);
        run = 0.0;
        nh++;
      }
      if (nh) run += p[k];
      else pre += p[k];
    }
  }
  const bool f = bits != 0;
  const unsigned F = __ballot_sync(FULL, f);
  // segmented inclusive scan: lane l's window never reaches below `start`,
  // its segment's first lane
  const int start = 31 - __clz(F & ((lane == 31) ? FULL : ((2u << lane) - 1u)));  // -1 if none
  double I = f ? run : pre;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const double u = __shfl_up_sync(FULL, I, d);
    if ((int)lane - d >= start && (int)lane >= d) I += u;
  }
  double E = __shfl_up_sync(FULL, I, 1);
  if (lane == 0) E = 0.0;
  // the run open at my lane start ends at my first start
  if (f && (lane > 0 || !(bits & 1u) || st.carry)) emit(o, st, rb - 1u, E + pre);
  st.csum = __shfl_sync(FULL, I, 31);
  st.carry = true;
  st.rbase += tot;
}

__device__ __forceinline__ unsigned lanemask_le() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_le;" : "=r"(m));
  return m;
}

// The 4-slot batch without per-slot branches: a lane's leading piece (slots
// before its first row start) and trailing piece (from its last row start)
// are masked sums; only lanes holding two or more row starts (rows shorter
// than 4 slots) take the loop that writes the runs between them.
template <>
__device__ __forceinline__ void batch<4>(const double (&p)[4], const Words<4> &hw, Run &st, const seg::Out &o) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned q = lane >> 3, sh = 4u * (lane & 7u);
  const UIN w0 = hw.w.x, w1 = hw.w.y, w2 = hw.w.z, w3 = hw.w.w;
  const unsigned c0 = __popc(w0), c1 = c0 + __popc(w1), c2 = c1 + __popc(w2), tot = c2 + __popc(w3);
  const UIN myw = q == 0 ? w0 : q == 1 ? w1 : q == 2 ? w2 : w3;
  const unsigned before = q == 0 ? 0u : q == 1 ? c0 : q == 2 ? c1 : c2;
  const unsigned bits = (myw >> sh) & 0xFu;
  const UIN rb = st.rbase + before + __popc(myw & ((1u << sh) - 1u));  // row of my first start
  const int first = bits ? __ffs(bits) - 1 : 4;
  const int last = bits ? 31 - __clz(bits) : 4;
  double pre = 0.0, run = 0.0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    pre += (k < first) ? p[k] : 0.0;
    run += (k >= last) ? p[k] : 0.0;
  }
  if (__popc(bits) >= 2) {
    UIN r = rb;
    double acc = 0.0;
    bool open = false;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      if ((bits >> k) & 1u) {
        if (open) emit(o, st, r++, acc);
        acc = 0.0;
        open = true;
      }
      acc += open ? p[k] : 0.0;
    }
  }
  if (lane == 0 && st.carry) pre += st.csum;
  const bool f = bits != 0;
  const unsigned F = __ballot_sync(FULL, f) & lanemask_le();
  const int start = F ? 31 - __clz(F) : 0;  // my segment's first lane
  const int reach = (int)lane - start;      // lanes below me in my segment
  double I = f ? run : pre;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const double u = __shfl_up_sync(FULL, I, d);
    if (reach >= d) I += u;
  }
  double E = __shfl_up_sync(FULL, I, 1);
  if (lane == 0) E = 0.0;
  if (f && (lane > 0 || !(bits & 1u) || st.carry)) emit(o, st, rb - 1u, E + pre);
  st.csum = __shfl_sync(FULL, I, 31);
  st.carry = true;
  st.rbase += tot;
}

__device__ __forceinline__ void finish(const Run &st, const seg::Out &o) {
  if ((threadIdx.x & 31u) != 0) return;
  const UIN crow = st.rbase - 1u;
  const size_t sg = st.seg;
  if (crow == st.row_a) {
    o.rec_row[2 * sg] = crow;
    o.rec_sum[2 * sg] = st.csum;
    o.rec_row[2 * sg + 1] = NO_ROW;
    o.rec_sum[2 * sg + 1] = 0.0;
  } else {
    o.rec_row[2 * sg + 1] = crow;
    o.rec_sum[2 * sg + 1] = st.csum;
  }
}

// SPL consecutive values / columns of one lane, and the batch's bitmap words.
template <typename VT, int SPL>
struct Vals;
template <>
struct Vals<double, 4> {
  double2 a, b;
  __device__ __forceinline__ void get(const double *v, size_t s) {
    const double2 *q = reinterpret_cast<const double2 *>(v + s);
    a = ld_stream(q);
    b = ld_stream(q + 1);
  }
  __device__ __forceinline__ double operator[](int k) const { return k == 0 ? a.x : k == 1 ? a.y : k == 2 ? b.x : b.y; }
};
template <>
struct Vals<double, 2> {
  double2 a;
  __device__ __forceinline__ void get(const double *v, size_t s) { a = ld_stream(reinterpret_cast<const double2 *>(v + s)); }
  __device__ __forceinline__ double operator[](int k) const { return k == 0 ? a.x : a.y; }
};
template <>
struct Vals<float, 4> {
  float4 a;
  __device__ __forceinline__ void get(const float *v, size_t s) { a = ld_stream(reinterpret_cast<const float4 *>(v + s)); }
  __device__ __forceinline__ float operator[](int k) const { return k == 0 ? a.x : k == 1 ? a.y : k == 2 ? a.z : a.w; }
};
template <>
struct Vals<float, 2> {
  float2 a;
  __device__ __forceinline__ void get(const float *v, size_t s) { a = ld_stream(reinterpret_cast<const float2 *>(v + s)); }
  __device__ __forceinline__ float operator[](int k) const { return k == 0 ? a.x : a.y; }
};

template <int SPL>
struct Cols;
template <>
struct Cols<4> {
  uint4 c;
  __device__ __forceinline__ void get(const UIN *col, size_t s) { c = ld_stream(reinterpret_cast<const uint4 *>(col + s)); }
  __device__ __forceinline__ UIN operator[](int k) const { return k == 0 ? c.x : k == 1 ? c.y : k == 2 ? c.z : c.w; }
};
template <>
struct Cols<2> {
  uint2 c;
  __device__ __forceinline__ void get(const UIN *col, size_t s) { c = ld_stream(reinterpret_cast<const uint2 *>(col + s)); }
  __device__ __forceinline__ UIN operator[](int k) const { return k == 0 ? c.x : c.y; }
};

template <int SPL>
__device__ __forceinline__ void get_words(Words<SPL> &w, const UIN *heads, size_t batch_start);
template <>
__device__ __forceinline__ void get_words<4>(Words<4> &w, const UIN *heads, size_t b) {
  w.w = __ldg(reinterpret_cast<const uint4 *>(heads + (b >> 5)));
}
template <>
__device__ __forceinline__ void get_words<2>(Words<2> &w, const UIN *heads, size_t b) {
  w.w = __ldg(reinterpret_cast<const uint2 *>(heads + (b >> 5)));
}

template <typename VT, int SPL>
struct Slots {
  Vals<VT, SPL> v;
  Cols<SPL> c;
  Words<SPL> h;
  __device__ __forceinline__ void get(const VT *val, const UIN *col, const UIN *heads, size_t batch_start,
                                      unsigned lane) {
    v.get(val, batch_start + SPL * lane);
    c.get(col, batch_start + SPL * lane);
    get_words<SPL>(h, heads, batch_start);
  }
};

// Plain-load kernel: one segment per warp, batches of 32*SPL slots, the
// loads of the next PD batches in flight while the current one gathers x and
// reduces; MINB CTAs of 256 threads per SM bound the registers.
template <typename VT, int SPL, int PD, int MINB, int PF = 0>
__global__ void __launch_bounds__(256, MINB) stream_ldg(size_t nslots, size_t nslots_pad, size_t seg_slots,
                                                        size_t nseg, const VT *__restrict__ val,
                                                        const UIN *__restrict__ col, const UIN *__restrict__ heads,
                                                        const UIN *__restrict__ segh, const FPT *__restrict__ x,
                                                        seg::Out o) {
  pdl_trigger();
  constexpr int BT = 32 * SPL;
  const unsigned lane = threadIdx.x & 31u;
  const size_t segid = ((size_t)blockIdx.x * 256 + threadIdx.x) >> 5;
  if (segid >= nseg) return;
  const size_t s0 = segid * seg_slots;
  const size_t s1 = min(s0 + seg_slots, nslots_pad);
  const int nbat = (int)((s1 - s0) / BT);
  Run st;
  begin(st, o, segid, segh[segid], __ldg(heads + (s0 >> 5)));
  Slots<VT, SPL> buf[PD + 1];
#pragma unroll
  for (int k = 0; k < PD; k++)
    if (k < nbat) buf[k].get(val, col, heads, s0 + (size_t)k * BT, lane);
  if (PF > 0 && lane == 0) {  // the first PF batches' streams into L2
    const size_t pb = min((size_t)PF * BT, s1 - s0);
    tma::prefetch_l2(val + s0, (uint32_t)(pb * sizeof(VT)));
    tma::prefetch_l2(col + s0, (uint32_t)(pb * 4));
  }
  for (int j = 0; j < nbat; j += PD + 1) {
#pragma unroll
    for (int r = 0; r <= PD; r++) {
      const int jj = j + r;
      if (jj >= nbat) break;
      if (PF > 0 && lane == 0 && jj + PF < nbat) {  // keep PF batches ahead in L2
        const size_t pb = s0 + (size_t)(jj + PF) * BT;
        tma::prefetch_l2(val + pb, BT * sizeof(VT));
        tma::prefetch_l2(col + pb, BT * 4);
      }
      const int nx = jj + PD;
      Slots<VT, SPL> &cur = buf[r];
      if (PD == 0) cur.get(val, col, heads, s0 + (size_t)jj * BT, lane);
      else if (nx < nbat) buf[(r + PD) % (PD + 1)].get(val, col, heads, s0 + (size_t)nx * BT, lane);
      const size_t sl = s0 + (size_t)jj * BT + SPL * lane;
      double p[SPL];
#pragma unroll
      for (int k = 0; k < SPL; k++) p[k] = pk::prod<VT>(cur.v[k], ldg(x + cur.c[k]));
      if (sl + SPL > nslots) {
#pragma unroll
        for (int k = 0; k < SPL; k++)
          if (sl + k >= nslots) p[k] = 0.0;
      }
      batch<SPL>(p, cur.h, st, o);
    }
  }
  finish(st, o);
}

// Work-queue form: persistent warps take whole segments from a device
// counter (reset to 0 before each launch) until none is left, so the
// segments of many uneven matrices concatenated into one stream (a
// block-diagonal batch) are shared out dynamically.  The loop ends when the
// counter passes the segment count; nothing waits.
template <typename VT>
__global__ void __launch_bounds__(256, 6) stream_queue(size_t nslots, size_t nslots_pad, size_t seg_slots,
                                                       size_t nseg, const VT *__restrict__ val,
                                                       const UIN *__restrict__ col, const UIN *__restrict__ heads,
                                                       const UIN *__restrict__ segh, const FPT *__restrict__ x,
                                                       unsigned long long *queue, seg::Out o) {
  pdl_trigger();
  constexpr int SPL = 4, BT = 128;
  const unsigned lane = threadIdx.x & 31u;
  for (;;) {
    unsigned long long next = 0;
    if (lane == 0) next = atomicAdd(queue, 1ull);
    const size_t segid = (size_t)__shfl_sync(FULL, next, 0);
    if (segid >= nseg) break;
    const size_t s0 = segid * seg_slots;
    const size_t s1 = min(s0 + seg_slots, nslots_pad);
    const int nbat = (int)((s1 - s0) / BT);
    Run st;
    begin(st, o, segid, segh[segid], __ldg(heads + (s0 >> 5)));
    for (int j = 0; j < nbat; j++) {
      Slots<VT, SPL> cur;
      cur.get(val, col, heads, s0 + (size_t)j * BT, lane);
      const size_t sl = s0 + (size_t)j * BT + SPL * lane;
      double p[SPL];
#pragma unroll
      for (int k = 0; k < SPL; k++) p[k] = pk::prod<VT>(cur.v[k], ldg(x + cur.c[k]));
      if (sl + SPL > nslots) {
#pragma unroll
        for (int k = 0; k < SPL; k++)
          if (sl + k >= nslots) p[k] = 0.0;
      }
      batch<SPL>(p, cur.h, st, o);
    }
    finish(st, o);
  }
}

// The per-CTA x windows of wide::stream_wide's staged form (STG): CTA b
// copies x[tlo[b], tlo[b] + tlen[b]) into shared memory with one bulk copy
// (tlo, tlen even; tlo + tlen <= n rounded down to even; tlen <= cap).  A
// gather whose column falls in the window reads shared memory; any other
// column reads x through L1/L2, so the result does not depend on it.
struct XWin {
  int nwin;            // 1 when the plan has windows, else 0
  UIN cap;             // doubles of shared memory per CTA
  UIN n;               // rows (= columns)
  const UIN *tlo = nullptr;
  const UIN *tlen = nullptr;
  int *status = nullptr;  // ISPMV_ERR_TIMEOUT when the copy's wait gave up
};

// Reduced-byte streams (4 slots per lane, no prefetch, 6 CTAs/SM):
//   LO   FP32 values plus, in segments whose rows need it, a BF16 residual
//        lo-word per slot: value = hi + lo, multiplied by x in FP64.
//   D16  16-bit column deltas from a per-batch base column (cmeta[b]); a
//        batch whose span does not fit 16 bits has its u32 columns in `esc`
//        (cmeta[b] = ESCAPE | escape index).
struct Narrow {
  const uint16_t *col16;  // D16 deltas
  const UIN *cmeta;       // D16 per-batch base or escape index
  const UIN *esc;         // D16 escaped batches' columns (128 each)
  const uint16_t *lo16;   // LO residuals of flagged segments, compacted
  const UIN *lo_off;      // LO per-segment offset into lo16, or NO_ROW
};
constexpr UIN ESCAPE = 0x80000000u;

__device__ __forceinline__ double bf16_to_double(uint16_t h) { return (double)__uint_as_float((UIN)h << 16); }

template <typename VT, bool LO, bool D16>
__global__ void __launch_bounds__(256, 6) stream_narrow(size_t nslots, size_t nslots_pad, size_t seg_slots,
                                                        size_t nseg, const VT *__restrict__ val,
                                                        const UIN *__restrict__ col, const UIN *__restrict__ heads,
                                                        const UIN *__restrict__ segh, Narrow nw,
                                                        const FPT *__restrict__ x, seg::Out o) {
  pdl_trigger();
  constexpr int SPL = 4, BT = 128;
  const unsigned lane = threadIdx.x & 31u;
  const size_t segid = ((size_t)blockIdx.x * 256 + threadIdx.x) >> 5;
  if (segid >= nseg) return;
  const size_t s0 = segid * seg_slots;
  const size_t s1 = min(s0 + seg_slots, nslots_pad);
  const int nbat = (int)((s1 - s0) / BT);
  Run st;
  begin(st, o, segid, segh[segid], __ldg(heads + (s0 >> 5)));
  UIN lo_base = NO_ROW;
  if (LO) lo_base = __ldg(nw.lo_off + segid);
  for (int j = 0; j < nbat; j++) {
    const size_t b = s0 + (size_t)j * BT, sl = b + SPL * lane;
    Vals<VT, SPL> v;
    v.get(val, sl);
    UIN c[SPL];
    if (D16) {
      const UIN m = __ldg(nw.cmeta + (b >> 7));
      if (m & ESCAPE) {
        const uint4 e = ld_stream(reinterpret_cast<const uint4 *>(nw.esc + (size_t)(m & ~ESCAPE) * BT + SPL * lane));
        c[0] = e.x; c[1] = e.y; c[2] = e.z; c[3] = e.w;
      } else {
        const uint2 d = ld_stream(reinterpret_cast<const uint2 *>(nw.col16 + sl));
        c[0] = m + (d.x & 0xFFFFu); c[1] = m + (d.x >> 16); c[2] = m + (d.y & 0xFFFFu); c[3] = m + (d.y >> 16);
      }
    } else {
      const uint4 e = ld_stream(reinterpret_cast<const uint4 *>(col + sl));
      c[0] = e.x; c[1] = e.y; c[2] = e.z; c[3] = e.w;
    }
    Words<SPL> h;
    get_words<SPL>(h, heads, b);
    double p[SPL];
    if (LO && lo_base != NO_ROW) {
      const uint2 l = ld_stream(reinterpret_cast<const uint2 *>(nw.lo16 + lo_base + (sl - s0)));
      const uint16_t lw[4] = {(uint16_t)(l.x & 0xFFFFu), (uint16_t)(l.x >> 16), (uint16_t)(l.y & 0xFFFFu),
                              (uint16_t)(l.y >> 16)};
#pragma unroll
      for (int k = 0; k < SPL; k++) {
        const double xv = ldg(x + c[k]);
        p[k] = fma(bf16_to_double(lw[k]), xv, (double)v[k] * xv);  // residual corrected in FP64
      }
    } else {
#pragma unroll
      for (int k = 0; k < SPL; k++) p[k] = pk::prod<VT>(v[k], ldg(x + c[k]));
    }
    if (sl + SPL > nslots) {
#pragma unroll
      for (int k = 0; k < SPL; k++)
        if (sl + k >= nslots) p[k] = 0.0;
    }
    batch<SPL>(p, h, st, o);
  }
  finish(st, o);
}

// Staged kernel: persistent warps, each with a ring of STAGES stages of
// SSZ slots filled by 1D bulk copies (values, columns, bitmap).  Streams are
// padded to SS = 512 slots, so any SSZ dividing 512 fits them.
constexpr int SS = 512;

template <typename VT, int SSZ>
constexpr uint32_t stage_bytes() {
  return SSZ * sizeof(VT) + SSZ * 4 + SSZ / 8;
}

template <int WARPS, int STAGES, typename VT, int SSZ>
constexpr size_t smem_bytes() {
  return ((WARPS * STAGES * 8 + 127) / 128) * 128 + (size_t)WARPS * STAGES * stage_bytes<VT, SSZ>();
}

template <int SSZ>
__device__ __forceinline__ uint32_t seg_nst(size_t seg, size_t seg_slots, size_t nslots_pad) {
  const size_t s0 = seg * seg_slots;
  if (s0 >= nslots_pad) return 0;
  const size_t left = nslots_pad - s0;
  return (uint32_t)((left < seg_slots ? left : seg_slots) / SSZ);
}

template <typename VT, int WARPS, int STAGES, int SSZ>
__global__ void __launch_bounds__(WARPS * 32) stream_tma(size_t nslots, size_t nslots_pad, size_t seg_slots,
                                                         size_t nseg, const VT *__restrict__ val,
                                                         const UIN *__restrict__ col, const UIN *__restrict__ heads,
                                                         const UIN *__restrict__ segh, const FPT *__restrict__ x,
                                                         seg::Out o, int *status) {
  pdl_trigger();
  constexpr uint32_t VB = SSZ * sizeof(VT), CB = SSZ * 4, HB = SSZ / 8, STB = VB + CB + HB;
  constexpr int NB = SSZ / BATCH;  // batches per stage
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
  size_t pseg = gw, cseg = gw;
  uint32_t pst = 0, cst = 0;
  auto issue = [&](int s) {
    const size_t b = pseg * seg_slots + (size_t)pst * SSZ;
    unsigned char *dst = ring + (size_t)s * STB;
    tma::bar_expect_tx(&bars[s], STB);
    tma::bulk_g2s(dst, val + b, VB, &bars[s], pol);
    tma::bulk_g2s(dst + VB, col + b, CB, &bars[s], pol);
    tma::bulk_g2s(dst + VB + CB, heads + b / 32, HB, &bars[s], pol);
    if (++pst >= seg_nst<SSZ>(pseg, seg_slots, nslots_pad)) {
      pseg += GW;
      pst = 0;
    }
  };
  if (lane == 0)
    for (int s = 0; s < STAGES && pseg < nseg; s++) issue(s);
  Run st;
  uint32_t t = 0;
  bool gaveup = false;
  while (cseg < nseg) {
    const int s = (int)(t % STAGES);
    if (!tma::bar_wait(&bars[s], (t / STAGES) & 1u)) {
      if (lane == 0 && status) atomicCAS(status, 0, ISPMV_ERR_TIMEOUT);
      gaveup = true;
      break;
    }
    const unsigned char *stage = ring + (size_t)s * STB;
    const VT *sv = reinterpret_cast<const VT *>(stage);
    const UIN *sc = reinterpret_cast<const UIN *>(stage + VB);
    const UIN *shd = reinterpret_cast<const UIN *>(stage + VB + CB);
    const size_t b = cseg * seg_slots + (size_t)cst * SSZ;
    if (cst == 0) begin(st, o, cseg, segh[cseg], shd[0]);
    double p[NB][4];
    Words<4> hw[NB];
#pragma unroll
    for (int j = 0; j < NB; j++) {
      const int i0 = BATCH * j + 4 * (int)lane;
      const uint4 c = *reinterpret_cast<const uint4 *>(sc + i0);
      const UIN cc[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
      for (int k = 0; k < 4; k++) p[j][k] = pk::prod<VT>(sv[i0 + k], ldg(x + cc[k]));
      hw[j].w = *reinterpret_cast<const uint4 *>(shd + 4 * j);
    }
    __syncwarp();
    if (lane == 0 && pseg < nseg) {
      tma::fence_proxy_async();
      issue(s);
    }
#pragma unroll
    for (int j = 0; j < NB; j++) {
      const size_t sl = b + BATCH * j + 4 * lane;
      if (sl + 4 > nslots) {
#pragma unroll
        for (int k = 0; k < 4; k++)
          if (sl + k >= nslots) p[j][k] = 0.0;
      }
      batch<4>(p[j], hw[j], st, o);
    }
    if (++cst >= seg_nst<SSZ>(cseg, seg_slots, nslots_pad)) {
      finish(st, o);
      cseg += GW;
      cst = 0;
    }
    t++;
  }
  if (gaveup)
    for (int s = 0; s < STAGES; s++) (void)tma::bar_wait(&bars[s], ((t + s) / STAGES) & 1u);
}

}  // namespace sss
}  // namespace ispmv
