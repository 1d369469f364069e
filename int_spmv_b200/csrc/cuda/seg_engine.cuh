// seg_engine.cuh - deterministic segmented row reduction for slot streams.
//
// The AXT layouts (and the compacted one's CSR order) lay every row's slots
// out contiguously, so a warp that walks a contiguous range of "units" (an
// AXT tile, a tile column, or one slot) sees each row as one run of equal
// row ids.  A warp owns one segment of units and:
//   - writes every run that starts and ends inside its segment straight to
//     y (such a run is a whole row);
//   - records its first run (head) and last run (tail) - which may continue
//     into a neighbouring segment - as (row, partial) pairs;
// and a fix-up kernel then adds each row's partials in segment order and
// writes y.  No atomics: y is overwritten (beta = 0) or accumulated
// (beta = 1) deterministically, and every row is written exactly once.
#pragma once
#include "common.cuh"

namespace ispmv {
namespace seg {

struct State {
  UIN crow;       // row of the run still open at the end of the last batch
  double csum;    // its partial sum
  bool head_done; // the segment's first run has been recorded
};

struct Out {
  FPT *y;
  const UIN *rowmap;  // compressed -> real row (nullptr: identity)
  UIN *rec_row;       // 2 records per segment: [2s] head, [2s+1] tail
  double *rec_sum;
  int beta;
};

__device__ __forceinline__ UIN real_row(const Out &o, UIN r) { return o.rowmap ? o.rowmap[r] : r; }

__device__ __forceinline__ void write_row(const Out &o, UIN r, double v) {
  const UIN rr = real_row(o, r);
  o.y[rr] = o.beta ? v + o.y[rr] : v;
}

// One batch of 32 units, one per lane: `p` the unit's partial sum, `r` its
// row (NO_ROW when !live).  Live lanes form a prefix of the warp.
__device__ __forceinline__ void batch(double p, UIN r, bool live, State &st, const Out &o, size_t segid) {
  const unsigned lane = threadIdx.x & 31u;
  // a batch past the segment's last unit changes nothing (the open run stays open)
  if (!__any_sync(FULL, live)) return;
  const UIN rprev = __shfl_up_sync(FULL, r, 1);
  const bool head = (lane == 0) ? (r != st.crow) : (r != rprev);
  // Did the carried run end at the previous batch's last lane?
  const bool carry_done = __shfl_sync(FULL, (unsigned)head, 0) && st.crow != NO_ROW;
  if (carry_done) {
    if (!st.head_done) {
      if (lane == 0) { o.rec_row[2 * segid] = st.crow; o.rec_sum[2 * segid] = st.csum; }
      st.head_done = true;
    } else if (lane == 0) {
      write_row(o, st.crow, st.csum);
    }
  }
  if (lane == 0 && !head) p += st.csum;
  const double s = warp_seg_scan(p, head);
  const UIN rnext = __shfl_down_sync(FULL, r, 1);
  const bool nlive = __shfl_down_sync(FULL, (unsigned)live, 1) != 0;
  const bool is_end = lane < 31 && live && nlive && r != rnext;
  unsigned ends = __ballot_sync(FULL, is_end);
  if (!st.head_done && ends) {
    const unsigned first = __ffs(ends) - 1;
    if (lane == first) { o.rec_row[2 * segid] = r; o.rec_sum[2 * segid] = s; }
    ends &= ~(1u << first);
    st.head_done = true;
  }
  if ((ends >> lane) & 1u) write_row(o, r, s);
  const unsigned lives = __ballot_sync(FULL, live);
  const int last = lives ? 31 - __clz(lives) : 0;
  const UIN lr = __shfl_sync(FULL, r, last);
  const double ls = __shfl_sync(FULL, s, last);
  if (lives) { st.crow = lr; st.csum = ls; }
}

// Records the segment's open run: its head if no run was recorded yet,
// else its tail.
__device__ __forceinline__ void finish(const State &st, const Out &o, size_t segid) {
  if ((threadIdx.x & 31u) != 0) return;
  if (!st.head_done) {
    o.rec_row[2 * segid] = st.crow;
    o.rec_sum[2 * segid] = st.crow == NO_ROW ? 0.0 : st.csum;
    o.rec_row[2 * segid + 1] = NO_ROW;
    o.rec_sum[2 * segid + 1] = 0.0;
  } else {
    o.rec_row[2 * segid + 1] = st.crow;
    o.rec_sum[2 * segid + 1] = st.crow == NO_ROW ? 0.0 : st.csum;
  }
}

// Fix-up: record i writes its row if it is the row's last record, adding the
// row's earlier records (walking back).  Also zeroes (beta = 0) the rows
// that own no slot at all (rows of length 0).  Launched as a programmatic
// dependent of the main kernel where the stream allows it, so its launch
// overlaps the main kernel's last CTAs: griddepcontrol.wait then blocks until
// the main kernel has completed and its records and rows are visible (it
// returns at once for an ordinary launch).
__global__ void fixup(size_t nrec, const UIN *__restrict__ rec_row, const double *__restrict__ rec_sum,
                      const UIN *__restrict__ rowmap, const UIN *__restrict__ empty, size_t nempty,
                      FPT *__restrict__ y, int beta) {
  pdl_wait();
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nempty && !beta) y[empty[i]] = 0.0;
  if (i >= nrec) return;
  const UIN r = rec_row[i];
  if (r == NO_ROW) return;
  size_t j = i + 1;
  while (j < nrec && rec_row[j] == NO_ROW) j++;
  if (j < nrec && rec_row[j] == r) return;
  double total = rec_sum[i];
  for (size_t k = i; k-- > 0;) {
    const UIN rk = rec_row[k];
    if (rk == NO_ROW) continue;
    if (rk != r) break;
    total += rec_sum[k];
  }
  const UIN rr = rowmap ? rowmap[r] : r;
  y[rr] = beta ? total + y[rr] : total;
}

}  // namespace seg
}  // namespace ispmv
