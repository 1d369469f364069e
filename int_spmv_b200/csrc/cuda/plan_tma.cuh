// plan_tma.cuh - TMA-staged AXT NOC tileH in {4, 8, 16} kernel of the plan layer.
//
// Every warp is persistent and owns a ring of STAGES shared-memory stages;
// one stage holds 512 consecutive slots of the value stream, the same slots
// of the column stream and their per-tile-column rows (the reference's sec).  Lane 0 keeps STAGES-1 stages in
// flight with 1D bulk copies (cp.async.bulk, evict-first in L2 so that x
// stays resident), while the warp consumes the oldest stage: it loads its
// slots' values and columns from shared memory, issues all of the stage's x
// gathers at once (read-only path, L2), then reduces rows.
//
// Warps walk segments (contiguous slot ranges) in a grid-stride order; the
// row reduction of a segment writes complete rows to y and leaves two
// (row, partial) records for the rows that cross its ends (seg_engine.cuh).
#pragma once
#include "plan_kernels.cuh"
#include "tma.cuh"

namespace ispmv {
namespace tk {

constexpr int SS = 512;  // slots per stage

template <typename VT>
struct StageLayout {
  static constexpr uint32_t VB = SS * sizeof(VT);  // values
  static constexpr uint32_t CB = SS * 4;           // columns
};

// Task cursor over (segment, stage) in this warp's order.
struct Cursor {
  size_t seg;
  uint32_t st;
};

__device__ __forceinline__ uint32_t seg_nst(size_t seg, size_t seg_slots, size_t nslots_pad) {
  const size_t s0 = seg * seg_slots;
  const size_t left = nslots_pad - s0;
  const size_t n = left < seg_slots ? left : seg_slots;
  return (uint32_t)(n / SS);
}

__device__ __forceinline__ void advance(Cursor &c, size_t seg_slots, size_t nslots_pad, size_t GW) {
  if (++c.st >= seg_nst(c.seg, seg_slots, nslots_pad)) {
    c.seg += GW;
    c.st = 0;
  }
}

__device__ __forceinline__ void set_status(int *status, int v) {
  if (status) atomicCAS(status, 0, v);
}

// Shared memory: WARPS*STAGES mbarriers (rounded to 128 B), then each warp's ring.
template <int WARPS, int STAGES>
__device__ __forceinline__ uint64_t *warp_bars(unsigned char *smem, int wib) {
  return reinterpret_cast<uint64_t *>(smem) + wib * STAGES;
}
template <int WARPS, int STAGES>
__device__ __forceinline__ unsigned char *warp_ring(unsigned char *smem, int wib, uint32_t stage_bytes) {
  constexpr uint32_t bar_bytes = ((WARPS * STAGES * 8 + 127) / 128) * 128;
  return smem + bar_bytes + (size_t)wib * STAGES * stage_bytes;
}

// ------------------------------------------------ AXT NOC th in {4,8,16} ---
// Stage = 512/TH units; each lane holds 16 slots: slot 32m + lane is sub-row
// (32m + lane)/8 mod TH of tile (32m)/(8TH), column lane % 8.
template <typename VT, int TH, int WARPS, int STAGES>
__global__ void __launch_bounds__(WARPS * 32) nocn_tma(size_t nunits, size_t nslots_pad, size_t nseg, size_t seg_slots,
                                                       const VT *__restrict__ val, const UIN *__restrict__ col,
                                                       const UIN *__restrict__ urow, const FPT *__restrict__ x,
                                                       seg::Out o, int *status) {
  pdl_trigger();
  using L = StageLayout<VT>;
  constexpr int UPS = SS / TH;           // units per stage
  constexpr int TPS = SS / (8 * TH);     // tiles per stage
  constexpr int MPT = TH / 4;            // 32-slot steps per tile
  constexpr uint32_t UB = UPS * 4;
  constexpr uint32_t STB = L::VB + L::CB + UB;
  extern __shared__ __align__(128) unsigned char smem[];
  const int wib = threadIdx.x >> 5;
  const unsigned lane = threadIdx.x & 31u;
  uint64_t *bars = warp_bars<WARPS, STAGES>(smem, wib);
  unsigned char *ring = warp_ring<WARPS, STAGES>(smem, wib, STB);
  const size_t gw = (size_t)blockIdx.x * WARPS + wib, GW = (size_t)gridDim.x * WARPS;
  if (gw >= nseg) return;
  if (lane == 0) {
    for (int s = 0; s < STAGES; s++) tma::bar_init(&bars[s], 1);
    tma::fence_barrier_init();
  }
  __syncwarp();
  const uint64_t pol = tma::policy_evict_first();
  auto issue = [&](const Cursor &c, int s) {
    const size_t b = c.seg * seg_slots + (size_t)c.st * SS;
    unsigned char *dst = ring + (size_t)s * STB;
    tma::bar_expect_tx(&bars[s], STB);
    tma::bulk_g2s(dst, val + b, L::VB, &bars[s], pol);
    tma::bulk_g2s(dst + L::VB, col + b, L::CB, &bars[s], pol);
    tma::bulk_g2s(dst + L::VB + L::CB, urow + b / TH, UB, &bars[s], pol);
  };
  Cursor pc{gw, 0}, cc{gw, 0};
  int gaveup = 0;
  if (lane == 0) {
    for (int s = 0; s < STAGES && pc.seg < nseg; s++) {
      issue(pc, s);
      advance(pc, seg_slots, nslots_pad, GW);
    }
  }
  seg::State st{NO_ROW, 0.0, false};
  uint32_t t = 0;
  while (cc.seg < nseg) {
    const int s = (int)(t % STAGES);
    if (!tma::bar_wait(&bars[s], (t / STAGES) & 1u)) {
      set_status(status, ISPMV_ERR_TIMEOUT);
      gaveup = 1;
      break;
    }
    const unsigned char *stage = ring + (size_t)s * STB;
    const VT *sv = reinterpret_cast<const VT *>(stage);
    const UIN *sc = reinterpret_cast<const UIN *>(stage + L::VB);
    const UIN *su = reinterpret_cast<const UIN *>(stage + L::VB + L::CB);
    const size_t u0 = (cc.seg * seg_slots + (size_t)cc.st * SS) / TH;
    if (cc.st == 0) st = seg::State{NO_ROW, 0.0, false};
    double p[16];
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int i = 32 * m + (int)lane;
      p[m] = pk::prod<VT>(sv[i], ldg(x + sc[i]));
    }
    UIN r[UPS / 32];
#pragma unroll
    for (int k = 0; k < UPS / 32; k++) r[k] = su[32 * k + lane];
    __syncwarp();
    if (lane == 0 && pc.seg < nseg) {
      tma::fence_proxy_async();
      issue(pc, s);
      advance(pc, seg_slots, nslots_pad, GW);
    }
    // column sums per tile: lane (l % 8) column, summed over the tile's sub-rows
    double cs[TPS];
#pragma unroll
    for (int T = 0; T < TPS; T++) {
      double a = 0.0;
#pragma unroll
      for (int m = 0; m < MPT; m++) a += p[T * MPT + m];
      a += __shfl_xor_sync(FULL, a, 8);
      a += __shfl_xor_sync(FULL, a, 16);
      cs[T] = a;
    }
#pragma unroll
    for (int bt = 0; bt < UPS / 32; bt++) {
      double mine = 0.0;
#pragma unroll
      for (int q = 0; q < 4; q++)
        if ((lane >> 3) == (unsigned)q) mine = cs[4 * bt + q];
      const size_t u = u0 + 32 * bt + lane;
      const bool live = u < nunits;
      seg::batch(mine, live ? r[bt] : NO_ROW, live, st, o, cc.seg);
    }
    if (cc.st + 1 >= seg_nst(cc.seg, seg_slots, nslots_pad)) seg::finish(st, o, cc.seg);
    advance(cc, seg_slots, nslots_pad, GW);
    t++;
  }
  if (gaveup)
    for (int s = 0; s < STAGES; s++) (void)tma::bar_wait(&bars[s], ((t + s) / STAGES) & 1u);
}

template <int WARPS, int STAGES>
constexpr size_t smem_bytes(uint32_t stage_bytes) {
  return ((WARPS * STAGES * 8 + 127) / 128) * 128 + (size_t)WARPS * STAGES * stage_bytes;
}

}  // namespace tk
}  // namespace ispmv
