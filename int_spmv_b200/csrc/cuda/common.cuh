// common.cuh - shared host and device helpers of the int_spmv_b200 CUDA layer.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "intspmv.h"

#define ISPMV_API extern "C" __attribute__((visibility("default")))

namespace ispmv {

constexpr unsigned FULL = 0xffffffffu;
constexpr UIN NO_ROW = 0xffffffffu;  // row id of a slot that belongs to no row

// ---- host side ----------------------------------------------------------
// Records a CUDA error text for ispmv_last_error() and maps it to a status.
int cuda_status(cudaError_t e, const char *where);
// Counts one launch of a library kernel (for ispmv_launch_count()).
void count_launch(unsigned n = 1);
// Checks the launch just made on the calling thread.
int check_launch(const char *where);
// Name given to the calling thread's latest check_launch (a static string).
const char *last_launch();
// Records a library error text for ispmv_last_error() and returns `status`.
int fail(int status, const char *text);
inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }
// Number of SMs of the current device (cached per device).
int sm_count();

#define ISPMV_TRY(expr)                                   \
  do {                                                    \
    cudaError_t e__ = (expr);                             \
    if (e__ != cudaSuccess) return ispmv::cuda_status(e__, #expr); \
  } while (0)

// ---- device side --------------------------------------------------------
// Programmatic dependent launch: a main kernel lets the launch that follows
// it in the stream (the row fix-up, K1's reorder) start now; that kernel
// waits (pdl_wait) for the whole main grid and its writes before it reads
// anything.  Both are no-ops for ordinary launches.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Inclusive segmented sum over the 32 lanes of a warp.  `head` marks the
// first lane of each run; lanes of one run end up holding the running sum
// from the run's head to themselves.
__device__ __forceinline__ double warp_seg_scan(double v, bool head) {
  const unsigned lane = threadIdx.x & 31u;
  unsigned f = head ? 1u : 0u;
#pragma unroll
  for (unsigned d = 1; d < 32; d <<= 1) {
    const double vu = __shfl_up_sync(FULL, v, d);
    const unsigned fu = __shfl_up_sync(FULL, f, d);
    if (lane >= d) {
      if (!f) v += vu;
      f |= fu;
    }
  }
  return v;
}

// Read-only (non-coherent) loads that keep the L1 line: used for x.
template <typename T>
__device__ __forceinline__ T ldg(const T *p) { return __ldg(p); }

// Streaming loads (evict-first): the value / index streams are read once.
__device__ __forceinline__ double ld_stream(const double *p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float *p) { return __ldcs(p); }
__device__ __forceinline__ UIN ld_stream(const UIN *p) { return __ldcs(p); }
__device__ __forceinline__ uint16_t ld_stream(const uint16_t *p) { return __ldcs(p); }
__device__ __forceinline__ double2 ld_stream(const double2 *p) { return __ldcs(p); }
__device__ __forceinline__ float4 ld_stream(const float4 *p) { return __ldcs(p); }
__device__ __forceinline__ uint4 ld_stream(const uint4 *p) { return __ldcs(p); }
__device__ __forceinline__ float2 ld_stream(const float2 *p) { return __ldcs(p); }
__device__ __forceinline__ uint2 ld_stream(const uint2 *p) { return __ldcs(p); }

}  // namespace ispmv
