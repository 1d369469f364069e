// selftest.cu - exercises the bounded device wait that every staged kernel
// (stream_tma, nocn_tma, stream_wide_tma) uses on its mbarriers, on a
// barrier that nothing ever completes: the wait must give up after its
// limit, record ISPMV_ERR_TIMEOUT in a device status word and return, and
// the context must stay usable.  No fault, trap or endless loop is involved.
#include "tma.cuh"

using namespace ispmv;

namespace {

__global__ void wait_probe(int *status, unsigned long long *elapsed_ns) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    tma::bar_init(&bar, 1);  // one arrival expected; none ever comes
    tma::fence_barrier_init();
  }
  __syncthreads();
  const uint64_t t0 = tma::global_ns();
  const bool done = tma::bar_wait(&bar, 0);
  const uint64_t t1 = tma::global_ns();
  if (threadIdx.x == 0) {
    *status = done ? ISPMV_OK : ISPMV_ERR_TIMEOUT;
    *elapsed_ns = t1 - t0;
  }
}

}  // namespace

// Runs the probe on `stream` and returns its status (ISPMV_ERR_TIMEOUT when
// the bounded wait behaves as designed); *elapsed_ms gets the time the wait
// took before giving up.  Allocates and frees an 16-byte status block.
ISPMV_API int ispmv_selftest_bounded_wait(double *elapsed_ms, void *stream) {
  cudaStream_t s = as_stream(stream);
  void *d = nullptr;
  ISPMV_TRY(cudaMalloc(&d, 16));
  int *status = static_cast<int *>(d);
  unsigned long long *ns = reinterpret_cast<unsigned long long *>(static_cast<char *>(d) + 8);
  int st = ISPMV_OK;
  if (cudaMemsetAsync(d, 0xff, 16, s) == cudaSuccess) {
    wait_probe<<<1, 32, 0, s>>>(status, ns);
    st = check_launch("wait_probe");
    int hs = ISPMV_ERR_CUDA;
    unsigned long long hns = 0;
    if (!st && cudaMemcpyAsync(&hs, status, sizeof hs, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
        cudaMemcpyAsync(&hns, ns, sizeof hns, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
        cudaStreamSynchronize(s) == cudaSuccess) {
      st = hs;
      if (elapsed_ms) *elapsed_ms = (double)hns * 1e-6;
    } else if (!st) {
      st = cuda_status(cudaGetLastError(), "ispmv_selftest_bounded_wait");
    }
  } else {
    st = cuda_status(cudaGetLastError(), "ispmv_selftest_bounded_wait");
  }
  cudaFree(d);
  return st;
}
