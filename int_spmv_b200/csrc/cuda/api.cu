// api.cu - status codes, error text, launch accounting and library facts.
#include <atomic>
#include <cstdio>
#include <cstring>

#include "common.cuh"

namespace ispmv {
namespace {
thread_local char g_last_error[256] = "";
thread_local const char *g_last_launch = "";
std::atomic<unsigned long long> g_launches{0};
int g_sms[64] = {0};
}  // namespace

int cuda_status(cudaError_t e, const char *where) {
  std::snprintf(g_last_error, sizeof g_last_error, "%s: %s", where, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? ISPMV_ERR_OOM : ISPMV_ERR_CUDA;
}

int fail(int status, const char *text) {
  std::snprintf(g_last_error, sizeof g_last_error, "%s", text);
  return status;
}

void count_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int check_launch(const char *where) {
  count_launch();
  g_last_launch = where;
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ISPMV_OK : cuda_status(e, where);
}

const char *last_launch() { return g_last_launch; }

int sm_count() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return 148;
  if (!g_sms[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    g_sms[dev] = v;
  }
  return g_sms[dev];
}

}  // namespace ispmv

ISPMV_API const char *ispmv_version(void) { return "int_spmv_b200 0.1 (sm_100a)"; }

ISPMV_API const char *ispmv_status_string(int st) {
  switch (st) {
    case ISPMV_OK: return "ok";
    case ISPMV_ERR_ARG: return "invalid argument or malformed matrix";
    case ISPMV_ERR_OOM: return "out of memory";
    case ISPMV_ERR_CUDA: return "CUDA error";
    case ISPMV_ERR_TIMEOUT: return "bounded device wait timed out";
    case ISPMV_ERR_UNSUPPORTED: return "unsupported configuration";
    case ISPMV_ERR_OVERFLOW: return "32-bit length or index overflow";
    default: return "unknown status";
  }
}

ISPMV_API const char *ispmv_last_error(void) { return ispmv::g_last_error; }

ISPMV_API unsigned long long ispmv_launch_count(void) { return ispmv::g_launches.load(); }
