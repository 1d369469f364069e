// tmem.cuh - the lane-interleaved slot-stream SpMV with its value/column
// stream staged through tensor memory (TMEM).
//
// Why: on B200 the slot-stream kernels are bound by the L1/TEX data pipe,
// which serves both the coalesced value/column loads and the scattered x
// gathers.  Tensor memory has its own path to the registers: the stream goes
// global -> shared memory (one 1D bulk copy per block, cp.async.bulk, no
// multicast) -> TMEM (tcgen05.cp, read by the tensor-core datapath) ->
// registers (tcgen05.ld), and the L1/TEX pipe is left to the gathers.
//
// CTA: 4*H consumer warps, warp w reading TMEM lane quadrant w % 4 (lanes
// 32(w%4).. - the quadrant tcgen05.ld lets it address) in column half w / 4,
// plus one producer warp.  Consumer warp w owns segment 4H*cta + w and walks
// it in batches of 32*SPL slots; lane l holds slots b + SPL*l + k, as in
// stream_wide, and the row reduction is wide::batch.
//
// Block layout (built by the plan): block j of CTA c holds batch j of the
// CTA's 4H segments, half h (segments 4h..4h+3 of the CTA) as NCP sub-blocks
// of 4 KB after the NCP of half h-1, each the no-swizzle K-major
// canonical layout of a 128-row x 256-bit matrix that tcgen05.cp.128x256b
// copies to 8 TMEM columns of all 128 lanes: row r = 32q + l at byte
// (r/8)*256 + (r%8)*16 of the sub-block, its second 16 bytes 128 further
// (descriptor LBO = 128, SBO = 256).  Row r's words are lane r's batch:
// the SPL values (two words each for FP64) then the SPL columns.
//
// Pipeline: S stages.  full[s] (bulk copy landed in shared memory) ->
// producer issues the stage's tcgen05.cp into TMEM columns [s*W, s*W+W) and
// tcgen05.commit -> tfull[s] -> consumers tcgen05.ld, then arrive on
// tempty[s] -> the producer may copy into TMEM stage s again; it refills
// shared stage s once tfull[s] shows the copy out of it is done.  Every wait
// is bounded (tma::bar_wait); a wait that gives up records ISPMV_ERR_TIMEOUT,
// the CTA drains its own bulk copies and tensor copies (bounded) and frees
// its TMEM before it exits.
#pragma once
#include "wide.cuh"

namespace ispmv {
namespace tmemk {

constexpr int CW = 4;  // TMEM lane quadrants: consumer warps per column half

// 32-bit words per lane and batch, tcgen05.cp copies (8 words) per stage,
// bytes of one stage block
template <typename VT, int SPL>
constexpr int words() {
  return SPL * (int)(sizeof(VT) / 4) + SPL;
}
template <typename VT, int SPL>
constexpr int ncp() {
  return words<VT, SPL>() / 8;
}
template <typename VT, int SPL>
constexpr uint32_t block_bytes() {
  return (uint32_t)ncp<VT, SPL>() * 4096u;
}
// TMEM columns allocated: a power of two >= 32 covering S stages
// H column halves: consumer warps 4h..4h+3 read TMEM columns [h*W, h*W+W)
// of each stage, so a CTA runs 4*H consumer warps.
template <typename VT, int SPL, int S, int H>
constexpr uint32_t tmem_cols() {
  uint32_t c = 32;
  while (c < (uint32_t)(S * H * words<VT, SPL>())) c *= 2;
  return c;
}
template <typename VT, int SPL, int S, int H>
constexpr size_t smem_bytes() {
  return (size_t)S * H * block_bytes<VT, SPL>();
}

// Word offset, in a stage block, of lane-row r's word m.
__host__ __device__ inline size_t blk_word(unsigned r, unsigned m) {
  const unsigned k = m / 8, w = m % 8, c = w / 4;
  return (size_t)k * 1024u + ((r / 8u) * 256u + c * 128u + (r % 8u) * 16u) / 4u + (w % 4u);
}

__device__ __forceinline__ uint64_t cp_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)(128u >> 4) << 16;  // leading byte offset: the row's second 16 bytes
  d |= (uint64_t)(256u >> 4) << 32;  // stride byte offset: the next 8 rows
  d |= (uint64_t)1 << 46;            // descriptor version of sm_100; no swizzle, base offset 0
  return d;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void bar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tma::smem_addr(bar)) : "memory");
}

// 8 TMEM columns of this warp's 32 lanes into 8 registers.
__device__ __forceinline__ void ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}

template <typename VT, typename XT, int SPL, int S, int H>
__global__ void __launch_bounds__((CW * H + 1) * 32)
    stream_tmem(size_t nslots, size_t seg_slots, const uint32_t *__restrict__ blocks, const UIN *__restrict__ heads,
                const UIN *__restrict__ segh, const XT *__restrict__ x, seg::Out o, int *status) {
  pdl_trigger();
  constexpr int BT = 32 * SPL, W = words<VT, SPL>(), NCP = ncp<VT, SPL>(), NW = CW * H;
  constexpr uint32_t BB = block_bytes<VT, SPL>() * H, TCOLS = tmem_cols<VT, SPL, S, H>();
  constexpr unsigned MASK = SPL == 32 ? 0xffffffffu : (1u << SPL) - 1u;
  static_assert(W % 8 == 0, "a lane's batch fills whole 8-column copies");
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[S], tfull[S], tempty[S];
  __shared__ uint32_t tbase;
  __shared__ int failed;
  const int warp = threadIdx.x >> 5;
  const unsigned lane = threadIdx.x & 31u;
  const int nbat = (int)(seg_slots / BT);  // every segment is full: the plan pads the stream to 4H segments per CTA
  if (warp == NW) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tma::smem_addr(&tbase)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; s++) {
      tma::bar_init(&full[s], 1);
      tma::bar_init(&tfull[s], 1);
      tma::bar_init(&tempty[s], NW);
    }
    failed = 0;
    tma::fence_barrier_init();
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tb = tbase;
  if (warp == NW) {
    if (lane == 0) {
      // producer
      const char *gblk = reinterpret_cast<const char *>(blocks) + (size_t)blockIdx.x * nbat * BB;
      const uint64_t pol = tma::policy_evict_first();
      const uint32_t sbase = tma::smem_addr(smem);
      int copied = 0, landed = 0, cped = 0;  // bulk copies issued and waited for, tensor copies committed
      for (int j = 0; j < S && j < nbat; j++, copied++) {
        tma::bar_expect_tx(&full[j], BB);
        tma::bulk_g2s(smem + (size_t)j * BB, gblk + (size_t)j * BB, BB, &full[j], pol);
      }
      bool ok = true;
      for (int j = 0; j < nbat && ok; j++) {
        const int s = j % S;
        const uint32_t ph = (uint32_t)(j / S) & 1u;
        ok = tma::bar_wait(&full[s], ph);
        if (!ok) break;
        landed++;
        ok = j < S || tma::bar_wait(&tempty[s], (uint32_t)((j - S) / S) & 1u);
        if (!ok) break;
        fence_after();
#pragma unroll
        for (int h = 0; h < H; h++)
#pragma unroll
          for (int k = 0; k < NCP; k++) {
            const uint64_t d = cp_desc(sbase + (uint32_t)(s * BB + (h * NCP + k) * 4096));
            asm volatile("tcgen05.cp.cta_group::1.128x256b [%0], %1;" ::"r"(tb + (uint32_t)((s * H + h) * W + 8 * k)),
                         "l"(d));
          }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         tma::smem_addr(&tfull[s]))
                     : "memory");
        cped++;
        if (j + S < nbat) {  // refill this shared stage once the tensor copy has read it
          ok = tma::bar_wait(&tfull[s], ph);
          if (!ok) break;
          tma::bar_expect_tx(&full[s], BB);
          tma::bulk_g2s(smem + (size_t)s * BB, gblk + (size_t)(j + S) * BB, BB, &full[s], pol);
          copied++;
        }
      }
      if (!ok) {
        atomicExch(&failed, 1);
        if (status) atomicCAS(status, 0, ISPMV_ERR_TIMEOUT);
        // drain: the bulk copies not yet waited for (at most one per stage)
        // and the last tensor copies land before the CTA frees its memory
        for (int j = landed; j < copied; j++) (void)tma::bar_wait(&full[j % S], (uint32_t)(j / S) & 1u);
        for (int j = cped > S ? cped - S : 0; j < cped; j++) (void)tma::bar_wait(&tfull[j % S], (uint32_t)(j / S) & 1u);
      }
    }
  } else {
    // consumer warp `warp`: segment NW*cta + warp, TMEM quadrant warp % 4,
    // column half warp / 4
    const size_t segid = (size_t)blockIdx.x * NW + warp;
    const size_t s0 = segid * seg_slots;
    sss::Run st;
    sss::begin(st, o, segid, segh[segid], __ldg(heads + (s0 >> 5)));
    const uint32_t tq = tb + ((uint32_t)(32 * (warp % CW)) << 16) + (uint32_t)((warp / CW) * W);
    bool ok = true;
    for (int j = 0; j < nbat; j++) {
      const int s = j % S;
      const uint32_t ph = (uint32_t)(j / S) & 1u;
      ok = __all_sync(FULL, tma::bar_wait(&tfull[s], ph)) && !*(volatile int *)&failed;
      if (!ok) break;
      fence_after();
      uint32_t wv[W];
#pragma unroll
      for (int k = 0; k < W / 8; k++) {
        uint32_t r8[8];
        ld8(tq + (uint32_t)(s * H * W + 8 * k), r8);
#pragma unroll
        for (int i = 0; i < 8; i++) wv[8 * k + i] = r8[i];
      }
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      fence_before();
      __syncwarp();
      if (lane == 0) bar_arrive(&tempty[s]);  // this warp's lanes of TMEM stage s are read
      const size_t b = s0 + (size_t)j * BT;
      const unsigned bits = (__ldg(heads + (b >> 5) + ((SPL * lane) >> 5)) >> ((SPL * lane) & 31u)) & MASK;
      VT v[SPL];
      XT xv[SPL];
#pragma unroll
      for (int k = 0; k < SPL; k++) {
        if constexpr (sizeof(VT) == 8) v[k] = __hiloint2double((int)wv[2 * k + 1], (int)wv[2 * k]);
        else v[k] = __uint_as_float(wv[k]);
        const UIN c = wv[(int)(sizeof(VT) / 4) * SPL + k];
        xv[k] = __ldg(x + c);
      }
      const size_t sl = b + (size_t)SPL * lane;
      if (sl + SPL > nslots) {  // the stream's zero padding adds nothing, whatever x holds
#pragma unroll
        for (int k = 0; k < SPL; k++)
          if (sl + k >= nslots) xv[k] = (XT)0;
      }
      wide::batch<VT, XT, SPL>(v, xv, bits, st, o);
    }
    if (ok) sss::finish(st, o);
    else if (lane == 0) atomicExch(&failed, 1);
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == NW) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tb), "r"(TCOLS));
}

}  // namespace tmemk
}  // namespace ispmv
