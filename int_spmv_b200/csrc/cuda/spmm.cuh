// spmm.cuh - multi-RHS SpMM on the slot stream: Y = A X, X and Y row-major
// n x k (FP64), one plan's slot stream read once for all k right-hand sides.
//
// A warp splits into 32/G groups of G lanes; lane jl of a group owns the W
// columns j0 + W*jl .. of the current column block (G*W = 8, 16 or 32
// columns).  Each group walks its own contiguous part of the warp's segment:
// G slots' values and columns are loaded per step (one per lane, coalesced)
// and broadcast with shuffles, each lane reads its W-wide piece of row
// X[col] (the group reads a contiguous row piece of X) and accumulates.
// Row starts come from the
// stream's bitmap; a row that ends inside the group's part is written to Y
// directly, the runs open at the part's two ends become G-wide records that
// spmm_fixup adds per row.  Deterministic, no atomics.  SPL > 0 reads a
// plan whose values and columns are stored lane-interleaved for stream_wide
// (wide::il_pos_c with SPL slots per lane); SPL = 0 a plan in slot order.
#pragma once
#include "wide.cuh"

namespace ispmv {
namespace mm {

struct Out {
  FPT *Y;
  const UIN *rowmap;
  UIN *rec_row;     // 2 per part
  double *rec_sum;  // 2 * G per part
  UIN k, j0, kb;    // row stride, first column of the block, columns in the block
};

__device__ __forceinline__ UIN real_row(const Out &o, UIN r) { return o.rowmap ? o.rowmap[r] : r; }

template <bool B>
struct BoolC {
  static constexpr bool value = B;
};

// One slot of a step as the group reads it from shared memory: its value
// and the column of the slot at the same place in the next step.
struct alignas(16) SlotRec {
  double v;
  UIN c, pad;
};

// G lanes per group, W (1 or 2) consecutive right-hand sides per lane: a
// pass covers CB = G*W columns.  A step of the group covers T = G slots:
// each lane loads one slot's value and column (coalesced), one step ahead
// of their use, and the group then works through the step's slots (8 at a
// time when G = 16) in two phases:
// first the X rows of all 8 slots are loaded into registers (W-wide vector
// loads of the group's contiguous piece of each row), then the row starts
// are handled and the products accumulated.  The loads of a step are thus in
// flight together, ahead of the stores that row ends make to Y, and the
// values and columns of the next step arrive meanwhile.
template <int G, int W, typename VT, int SPL>
__global__ void __launch_bounds__(256) stream_spmm(size_t nslots, size_t nslots_pad, size_t seg_slots, size_t nseg,
                                                   const VT *__restrict__ val, const UIN *__restrict__ col,
                                                   const UIN *__restrict__ heads, const UIN *__restrict__ segh,
                                                   const FPT *__restrict__ X, Out o) {
  static_assert(W == 1 || W == 2, "one or two right-hand sides per lane");
  constexpr int NG = 32 / G;            // groups per warp = parts per segment
  constexpr int CB = G * W;             // columns of one pass
  constexpr int R = 1;                  // slots per lane and step
  constexpr int T = G * R;              // slots per step (4, 8 or 16: within one bitmap word)
  constexpr int SUB = T < 8 ? T : 8;    // slots whose X rows are loaded together
  const unsigned lane = threadIdx.x & 31u, grp = lane / G, jl = lane % G;
  const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (grp * G));
  const size_t segid = ((size_t)blockIdx.x * 256 + threadIdx.x) >> 5;
  if (segid >= nseg) return;
  const size_t s0 = segid * seg_slots;
  const size_t seg_end = min(s0 + seg_slots, nslots_pad);
  const size_t part = (seg_end - s0) / NG;  // a multiple of 32
  const size_t a = s0 + grp * part, b = a + part;
  const size_t pid = segid * NG + grp;
  // compressed row of the run open at slot a: starts before a, minus one
  UIN cr = segh[segid];
  for (size_t w = s0 >> 5; w < (a >> 5); w++) cr += __popc(__ldg(heads + w));
  const bool a_head = (__ldg(heads + (a >> 5)) & 1u) != 0;  // a is 32-aligned
  const UIN row_a = a_head ? NO_ROW : cr - 1u;
  UIN row = cr - 1u;    // current run's row (advanced at each start)
  bool have = !a_head;  // the current run has slots in this part
  const unsigned j = jl * W;  // my first column in the block
  const int ncol = j < o.kb ? min(W, (int)(o.kb - j)) : 0;  // my live columns (0..W)
  // W-wide loads and stores need 16-byte rows: k even, j0 even, X and Y aligned
  const bool vec = W == 2 && ncol == 2 && ((o.k | o.j0) & 1u) == 0 &&
                   ((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(o.Y)) & 15u) == 0;
  const size_t xoff = o.j0 + j;
  double acc[W];
#pragma unroll
  for (int w = 0; w < W; w++) acc[w] = 0.0;
  if (jl == 0) {
    o.rec_row[2 * pid] = NO_ROW;
    o.rec_row[2 * pid + 1] = NO_ROW;
  }
#pragma unroll
  for (int w = 0; w < W; w++) {
    if (w < ncol) {
      o.rec_sum[(2 * pid) * CB + j + w] = 0.0;
      o.rec_sum[(2 * pid + 1) * CB + j + w] = 0.0;
    }
  }
  auto put = [&](UIN r) {  // the run of row r ends: Y or the part's head record
#pragma unroll
    for (int w = 0; w < W; w++) {
      if (w < ncol) {
        if (r == row_a) o.rec_sum[(2 * pid) * CB + j + w] = acc[w];
        else o.Y[(size_t)real_row(o, r) * o.k + xoff + w] = acc[w];
      }
    }
  };
  // the step's slots: lane jl holds slots c0 + q*G + jl, q < R
  VT nv[R];
  UIN nc[R], nhw = 0;
  auto load_step = [&](size_t c0) {
#pragma unroll
    for (int q = 0; q < R; q++) {
      const size_t my = c0 + (size_t)q * G + jl;
      nv[q] = val[wide::il_pos_c<SPL, 16u / sizeof(VT)>(my)];
      nc[q] = col[wide::il_pos_c<SPL, 4u>(my)];
    }
    nhw = __ldg(heads + (c0 >> 5));
  };
  if (a < b) load_step(a);
  for (size_t c0 = a; c0 < b; c0 += T) {
    VT mv[R];
    UIN mc[R];
#pragma unroll
    for (int q = 0; q < R; q++) {
      mv[q] = nv[q];
      mc[q] = nc[q];
    }
    const UIN hw = nhw;
    if (c0 + T < b) load_step(c0 + T);
#pragma unroll
    for (int i0 = 0; i0 < T; i0 += SUB) {
      double xv[SUB][W];
      double vv[SUB];
#pragma unroll
      for (int u = 0; u < SUB; u++) {
        const int i = i0 + u;  // slot c0 + i: lane i % G, register i / G
        vv[u] = (double)__shfl_sync(gmask, mv[i / G], grp * G + i % G);
        const UIN c = __shfl_sync(gmask, mc[i / G], grp * G + i % G);
        const bool live = c0 + i < nslots;
        const FPT *xr = X + (size_t)c * o.k + xoff;
        if (vec) {
          const double2 qx = live ? __ldg(reinterpret_cast<const double2 *>(xr)) : make_double2(0.0, 0.0);
          xv[u][0] = qx.x;
          xv[u][W - 1] = qx.y;
        } else {
#pragma unroll
          for (int w = 0; w < W; w++) xv[u][w] = (live && w < ncol) ? __ldg(xr + w) : 0.0;
        }
      }
#pragma unroll
      for (int u = 0; u < SUB; u++) {
        const size_t s = c0 + i0 + u;
        if ((hw >> (s & 31u)) & 1u) {  // a row starts at s: the current run ends
          if (have) {
            if (vec && row != row_a) {
              *reinterpret_cast<double2 *>(o.Y + (size_t)real_row(o, row) * o.k + xoff) =
                  make_double2(acc[0], acc[W - 1]);
            } else {
              put(row);
            }
            if (row == row_a && jl == 0) o.rec_row[2 * pid] = row;
          }
          row++;
#pragma unroll
          for (int w = 0; w < W; w++) acc[w] = 0.0;
          have = true;
        }
#pragma unroll
        for (int w = 0; w < W; w++) acc[w] = fma(vv[u], xv[u][w], acc[w]);
      }
    }
  }
  // the run open at the part's end
  if (have) {
    const bool is_a = row == row_a;
    if (jl == 0) o.rec_row[2 * pid + (is_a ? 0 : 1)] = row;
#pragma unroll
    for (int w = 0; w < W; w++)
      if (w < ncol) o.rec_sum[(2 * pid + (is_a ? 0 : 1)) * CB + j + w] = acc[w];
  }
}

// 32-byte global accesses (sm_100): four consecutive doubles, the address
// 32-byte aligned.
__device__ __forceinline__ void ld4(const double *p, double (&d)[4]) {
  asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
               : "=d"(d[0]), "=d"(d[1]), "=d"(d[2]), "=d"(d[3])
               : "l"(p));
}
__device__ __forceinline__ void st4(double *p, const double (&d)[4]) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(d[0]), "d"(d[1]), "d"(d[2]), "d"(d[3])
               : "memory");
}

// Four right-hand sides per lane: a group of G lanes covers CB = 4G columns
// (8, 16 or 32) with one 32-byte X load per lane and slot, and NG = 32 / G
// groups per warp each walk their own part of the segment as in
// stream_spmm.  A step takes T slots of the group; its X row pieces are
// loaded while the step before is consumed, slot by slot, into the registers
// that slot of the step before has just freed, so every lane keeps T loads
// in flight all the time (not T at the start of a step and none while it is
// consumed).  Values and columns of step s+1 are in registers during step
// s, and those of step s+2 are loaded at its start; at a step's start each
// lane writes its slots' values and next columns to the warp's records in
// shared memory, which the group then reads as broadcasts.  Needs k and j0
// multiples of 4 and X and Y 32-byte aligned (kb is then a multiple of 4
// too); lanes past the block's last column load a piece of the block and
// store nothing.  The last step of a part is compiled apart (no loads for a
// next step), so a slot costs no test for it.
template <int G, int T, int MINB, typename VT, int SPL>
__global__ void __launch_bounds__(256, MINB)
    stream_spmm4(size_t nslots, size_t nslots_pad, size_t seg_slots, size_t nseg, const VT *__restrict__ val,
                 const UIN *__restrict__ col, const UIN *__restrict__ heads, const UIN *__restrict__ segh,
                 const FPT *__restrict__ X, Out o) {
  static_assert(T % G == 0 && T <= 32 && 32 % T == 0, "a step is whole lanes and inside one bitmap word");
  constexpr int W = 4, NG = 32 / G, CB = G * W, R = T / G;  // R: slots per lane whose value and column it loads
  const unsigned lane = threadIdx.x & 31u, grp = lane / G, jl = lane % G;
  const size_t segid = ((size_t)blockIdx.x * 256 + threadIdx.x) >> 5;
  if (segid >= nseg) return;
  const size_t s0 = segid * seg_slots;
  const size_t seg_end = min(s0 + seg_slots, nslots_pad);
  const size_t part = (seg_end - s0) / NG;  // a multiple of 32
  const size_t a = s0 + grp * part, b = a + part;
  const size_t pid = segid * NG + grp;
  UIN cr = segh[segid];
  for (size_t w = s0 >> 5; w < (a >> 5); w++) cr += __popc(__ldg(heads + w));
  const bool a_head = (__ldg(heads + (a >> 5)) & 1u) != 0;
  const UIN row_a = a_head ? NO_ROW : cr - 1u;
  UIN row = cr - 1u;
  bool have = !a_head;
  const unsigned j = jl * W;
  const bool live = j < o.kb;  // all four columns, or none
  const FPT *xb = X + o.j0 + (live ? j : o.kb - W);
  double acc[W] = {0.0, 0.0, 0.0, 0.0};
  if (jl == 0) {
    o.rec_row[2 * pid] = NO_ROW;
    o.rec_row[2 * pid + 1] = NO_ROW;
  }
  if (live) {
#pragma unroll
    for (int w = 0; w < W; w++) {
      o.rec_sum[(2 * pid) * CB + j + w] = 0.0;
      o.rec_sum[(2 * pid + 1) * CB + j + w] = 0.0;
    }
  }
  auto load_step = [&](size_t c0, VT (&lv)[R], UIN (&lc)[R], UIN &lw) {
#pragma unroll
    for (int q = 0; q < R; q++) {
      const size_t my = c0 + (size_t)q * G + jl;
      lv[q] = val[wide::il_pos_c<SPL, 16u / sizeof(VT)>(my)];
      lc[q] = col[wide::il_pos_c<SPL, 4u>(my)];
    }
    lw = __ldg(heads + (c0 >> 5));
  };
  if (a >= b) return;
  // step s in registers: values mv, bitmap word mw, X pieces xv; step s+1:
  // values v1, columns c1, word w1; step s+2: v2, c2, w2 (in flight)
  VT mv[R], v1[R] = {}, v2[R] = {};
  UIN mc[R], c1[R] = {}, c2[R] = {}, mw, w1 = 0, w2 = 0;
  double xv[T][W];
  load_step(a, mv, mc, mw);
  if (a + T < b) load_step(a + T, v1, c1, w1);
#pragma unroll
  for (int i = 0; i < T; i++) {
    const UIN c = __shfl_sync(FULL, mc[i / G], grp * G + i % G);
    ld4(xb + (size_t)c * o.k, xv[i]);
  }
  // a run that ends is stored to its Y row, or to the part's head record
  // when it is the row open at the part's start (a select, not a branch);
  // lanes past the block's last column store nothing
  double *const head = o.rec_sum + (2 * pid) * CB + j;
  // the warp's slot records: group g's slot i at g * (T + 1) + i (one
  // record of padding per group, so the groups' broadcasts fall in
  // different banks)
  constexpr int RS = T + 1;
  __shared__ SlotRec recs[8][NG * RS];
  SlotRec *const wrec = recs[threadIdx.x >> 5];
  const SlotRec *const grec = wrec + grp * RS;
  auto step = [&](size_t c0, auto more_c) {
    constexpr bool MORE = decltype(more_c)::value;  // step s+1 exists: load its X pieces
#pragma unroll
    for (int q = 0; q < R; q++) wrec[grp * RS + q * G + jl] = SlotRec{(double)mv[q], c1[q], 0u};
    __syncwarp();
    if (c0 + 2 * T < b) load_step(c0 + 2 * T, v2, c2, w2);
    if (c0 + T > nslots) {  // the stream's zero padding adds nothing, whatever X holds
#pragma unroll
      for (int i = 0; i < T; i++)
        if (c0 + i >= nslots) {
#pragma unroll
          for (int w = 0; w < W; w++) xv[i][w] = 0.0;
        }
    }
    const unsigned hs = mw >> (unsigned)(c0 & 31u);
#pragma unroll
    for (int i = 0; i < T; i++) {
      const SlotRec sr = grec[i];
      const double v = sr.v;
      if (hs & (1u << i)) {  // a row starts at slot c0 + i: the current run ends
        const bool is_a = row == row_a;
        double *dst = is_a ? head : o.Y + (size_t)real_row(o, row) * o.k + o.j0 + j;
        if (have && live) st4(dst, acc);
        if (have && is_a && jl == 0) o.rec_row[2 * pid] = row;
        row++;
#pragma unroll
        for (int w = 0; w < W; w++) acc[w] = 0.0;
        have = true;
      }
#pragma unroll
      for (int w = 0; w < W; w++) acc[w] = fma(v, xv[i][w], acc[w]);
      if constexpr (MORE) ld4(xb + (size_t)sr.c * o.k, xv[i]);  // slot i of step s+1, into the registers just freed
    }
    __syncwarp();  // every lane has read the records before the next step writes them
#pragma unroll
    for (int q = 0; q < R; q++) {
      mv[q] = v1[q];
      c1[q] = c2[q];
      v1[q] = v2[q];
    }
    mw = w1;
    w1 = w2;
  };
  size_t c0 = a;
  for (; c0 + T < b; c0 += T) step(c0, BoolC<true>{});
  step(c0, BoolC<false>{});
  if (have) {  // the run open at the part's end
    const bool is_a = row == row_a;
    if (jl == 0) o.rec_row[2 * pid + (is_a ? 0 : 1)] = row;
    if (live) {
#pragma unroll
      for (int w = 0; w < W; w++) o.rec_sum[(2 * pid + (is_a ? 0 : 1)) * CB + j + w] = acc[w];
    }
  }
}

// Record i (of 2 per part) writes its row if it is that row's last record,
// adding the row's earlier records; rows with no slot get zeros.
template <int G>  // G = columns of one pass
__global__ void spmm_fixup(size_t nrec, const UIN *__restrict__ rec_row, const double *__restrict__ rec_sum,
                           const UIN *__restrict__ empty, size_t nempty, Out o) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t i = t / G;
  const unsigned j = t % G;
  if (j >= o.kb) return;
  if (i < nempty) o.Y[(size_t)empty[i] * o.k + o.j0 + j] = 0.0;
  if (i >= nrec) return;
  const UIN r = rec_row[i];
  if (r == NO_ROW) return;
  size_t q = i + 1;
  while (q < nrec && rec_row[q] == NO_ROW) q++;
  if (q < nrec && rec_row[q] == r) return;
  double total = rec_sum[i * G + j];
  for (size_t m = i; m-- > 0;) {
    const UIN rm = rec_row[m];
    if (rm == NO_ROW) continue;
    if (rm != r) break;
    total += rec_sum[m * G + j];
  }
  o.Y[(size_t)real_row(o, r) * o.k + o.j0 + j] = total;
}

}  // namespace mm
}  // namespace ispmv
