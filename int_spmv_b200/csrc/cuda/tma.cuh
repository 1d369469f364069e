// tma.cuh - 1D bulk copies (cp.async.bulk, the TMA engine's untiled form)
// into shared memory, completed on mbarriers, for per-warp staging rings.
//
// One lane of a warp owns the ring: it arms a stage's mbarrier with the
// byte count it expects and issues the bulk copies; every lane then waits on
// the stage's phase.  Waits are bounded: after WAIT_LIMIT polls the kernel
// records ISPMV_ERR_TIMEOUT in a device status word and gives up.
// No multicast: every copy reads this GPU's own memory into its own CTA.
#pragma once
#include <stdint.h>

#include "common.cuh"

namespace ispmv {
namespace tma {

constexpr uint32_t WAIT_LIMIT = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void bar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the async proxy (TMA).
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier shared-memory accesses (generic proxy)
// before later bulk copies (async proxy) into the same buffer.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void bar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

// dst (shared) <- src (global), `bytes` a multiple of 16, both 16-byte aligned.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                         uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

// The same copy with the default L2 policy (data other CTAs read again).
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

// Prefetches `bytes` (a multiple of 16, 16-byte aligned) of global memory
// into L2 through the bulk-copy engine; no registers or shared memory.
__device__ __forceinline__ void prefetch_l2(const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool bar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the phase with parity `parity`: at most WAIT_LIMIT polls
// and WAIT_NS nanoseconds; false = gave up.
constexpr uint64_t WAIT_NS = 200ull * 1000 * 1000;
__device__ __forceinline__ bool bar_wait(uint64_t *bar, uint32_t parity) {
  if (bar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t i = 1; i < WAIT_LIMIT; i++) {
    if (bar_try_wait(bar, parity)) return true;
    if ((i & 255u) == 0 && global_ns() - t0 > WAIT_NS) return false;
  }
  return false;
}

}  // namespace tma
}  // namespace ispmv
