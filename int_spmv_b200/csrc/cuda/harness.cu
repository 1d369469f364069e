// harness.cu - the reference's per-kernel harness (edoardoCB/int_spmv,
// intSpmv_main.c: test_cf_CSR :433, test_int_AXC :736, test_int_k1 :980,
// test_int_k1p :1070, test_int_axt_noc_h1 :1408, test_int_axt_noc :1478,
// test_int_axt_com_h1 :1570) on the GPU kernels of literal.cu.
//
// Each wrapper takes the reference's arrays (host memory, as its builders
// produce them), uploads them once, runs the kernel NUM_ITE times with a
// CUDA event pair around every launch, and returns the reference's str_res:
// its name string, the mean run time `et` in seconds, `ot` (the reorder pass
// of test_int_k1, else 0), flops = 2*nnz / et, and getErrors of the result
// against `ref`.  As in the reference, the AXT kernels accumulate into a y
// that is zeroed before every run, outside the timed region (M:1420, 1491,
// 1590), and any failure prints and exits.
//
// Compiled twice like literal.cu: FPT = double, and FPT = float with the
// `_f32` names (intspmv.h maps them).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"

using namespace ispmv;

#ifndef ISPMV_FPT_FLOAT
namespace {
volatile UIN g_num_ite = 0;  // 0: $ISPMV_NUM_ITE or the reference's default
}
ISPMV_API void ispmv_set_num_ite(UIN n) { g_num_ite = n; }
ISPMV_API UIN ispmv_get_num_ite(void) {
  const UIN n = g_num_ite;
  if (n) return n;
  if (const char *e = getenv("ISPMV_NUM_ITE")) {
    const long v = strtol(e, nullptr, 10);
    if (v > 0 && v < 1000000000L) return (UIN)v;
  }
  return ISPMV_NUM_ITE_DEFAULT;
}
#endif

namespace {

[[noreturn]] void die(const char *fn, int st) {
  fflush(stdout);
  printf("\n%s failed: %s (%s)\n", fn, ispmv_status_string(st), ispmv_last_error());
  fflush(stdout);
  exit(EXIT_FAILURE);
}

#define HCHK(expr)                 \
  do {                             \
    const int s__ = (expr);        \
    if (s__) die(fn, s__);         \
  } while (0)

// Device buffers and events of one harness call, released on every return.
struct Run {
  std::vector<void *> bufs;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ~Run() {
    for (void *p : bufs) cudaFree(p);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
  int events() {
    ISPMV_TRY(cudaEventCreate(&e0));
    ISPMV_TRY(cudaEventCreate(&e1));
    return ISPMV_OK;
  }
  template <typename T>
  int alloc(size_t n, T **d, bool zero = false) {
    void *p = nullptr;
    ISPMV_TRY(cudaMalloc(&p, (n ? n : 1) * sizeof(T)));
    bufs.push_back(p);
    if (zero && n) ISPMV_TRY(cudaMemset(p, 0, n * sizeof(T)));
    *d = static_cast<T *>(p);
    return ISPMV_OK;
  }
  template <typename T>
  int up(const T *h, size_t n, T **d) {
    int st = alloc(n, d);
    if (st) return st;
    if (n) {
      if (!h) return fail(ISPMV_ERR_ARG, "test_*: a host array of the format is null");
      ISPMV_TRY(cudaMemcpy(*d, h, n * sizeof(T), cudaMemcpyHostToDevice));
    }
    return ISPMV_OK;
  }
  // Mean seconds of `iters` runs of launch(); clear() (if given) runs before
  // each, outside the event pair.
  template <typename L, typename C>
  int time(UIN iters, L &&launch, C &&clear, double *mean_s) {
    double total_ms = 0.0;
    for (UIN i = 0; i < iters; i++) {
      int st = clear();
      if (st) return st;
      ISPMV_TRY(cudaEventRecord(e0, nullptr));
      st = launch();
      if (st) return st;
      ISPMV_TRY(cudaEventRecord(e1, nullptr));
      ISPMV_TRY(cudaEventSynchronize(e1));
      float ms = 0.0f;
      ISPMV_TRY(cudaEventElapsedTime(&ms, e0, e1));
      total_ms += ms;
    }
    *mean_s = iters ? total_ms / 1e3 / iters : 0.0;
    return ISPMV_OK;
  }
};

auto no_clear = [] { return ISPMV_OK; };

int zero(FPT *y, size_t bytes) {
  const cudaError_t e = cudaMemsetAsync(y, 0, bytes, nullptr);
  return e == cudaSuccess ? ISPMV_OK : cuda_status(e, "test_*: zero y");
}

str_res make_res(const char *name, double et, double ot, UIN nnz) {
  str_res sr;
  memset(&sr, 0, sizeof sr);
  const size_t len = strnlen(name, sizeof sr.name - 1);  // the reference's names fit its 25 bytes
  memcpy(sr.name, name, len);
  sr.name[len] = '\0';
  sr.et = et;
  sr.ot = ot;
  sr.flops = et > 0.0 ? 2.0 * (double)nnz / et : 0.0;
  return sr;
}

// The result back on the host, then getErrors against ref (M:404-425).
void finish(const char *fn, str_res *sr, const FPT *d_res, UIN n, const FPT *ref) {
  std::vector<FPT> h(n ? n : 1);
  if (n) {
    const cudaError_t e = cudaMemcpy(h.data(), d_res, (size_t)n * sizeof(FPT), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) die(fn, cuda_status(e, "test_*: result copy"));
  }
  getErrors(n, ref, h.data(), &sr->sErr);
}

}  // namespace

ISPMV_API str_res test_cf_CSR(const str_matCSR matCSR, const FPT *vec, const FPT *ref) {
  const char *fn = "test_cf_CSR";
  const UIN n = matCSR.nrows, nnz = matCSR.nnz;
  Run r;
  UIN *row, *col;
  FPT *val, *x, *y;
  HCHK(r.events());
  HCHK(r.up(matCSR.row, (size_t)n + 1, &row));
  HCHK(r.up(matCSR.col, nnz, &col));
  HCHK(r.up(matCSR.val, nnz, &val));
  HCHK(r.up(vec, n, &x));
  HCHK(r.alloc(n, &y, true));
  double et = 0.0;
  HCHK(r.time(ispmv_get_num_ite(), [&] { return ispmv_dev_cf_csr(n, row, col, val, x, y, nullptr); }, no_clear, &et));
  str_res sr = make_res("cf_CSR", et, 0.0, nnz);
  finish(fn, &sr, y, n, ref);
  return sr;
}

ISPMV_API str_res test_int_AXC(const UIN ompNT, const str_matAXC matAXC, const FPT *ref) {
  const char *fn = "test_int_AXC";
  (void)ompNT;
  const UIN n = matAXC.nrows;
  Run r;
  UIN *brp;
  FPT *ax, *y;
  HCHK(r.events());
  HCHK(r.up(matAXC.brp, (size_t)n + 1, &brp));
  HCHK(r.up(matAXC.ax, matAXC.lenAX, &ax));
  HCHK(r.alloc(n, &y, true));
  double et = 0.0;
  HCHK(r.time(ispmv_get_num_ite(), [&] { return ispmv_dev_int_axc(n, ax, brp, y, nullptr); }, no_clear, &et));
  str_res sr = make_res("int_AXC", et, 0.0, matAXC.nnz);
  finish(fn, &sr, y, n, ref);
  return sr;
}

namespace {
struct K1Dev {
  FPT *val, *x;
  UIN *col, *chp, *nmc, *permi;
};
int upload_k1(Run &r, const str_matK1 &m, const FPT *vec, K1Dev *d) {
  int st;
  if ((st = r.up(m.val, m.lenVC, &d->val))) return st;
  if ((st = r.up(m.col, m.lenVC, &d->col))) return st;
  if ((st = r.up(m.chp, m.chunkNum, &d->chp))) return st;
  if ((st = r.up(m.nmc, m.chunkNum, &d->nmc))) return st;
  if ((st = r.up(m.permi, (size_t)m.chunkNum * ISPMV_CHUNK_SIZE, &d->permi))) return st;
  return r.up(vec, m.nrows, &d->x);
}
}  // namespace

ISPMV_API str_res test_int_k1(const UIN ompNT, const str_matK1 matK1, const FPT *vec, const FPT *ref) {
  const char *fn = "test_int_k1";
  (void)ompNT;
  const UIN cn = matK1.chunkNum, n = matK1.nrows;
  Run r;
  K1Dev d;
  FPT *res, *ord;
  HCHK(r.events());
  HCHK(upload_k1(r, matK1, vec, &d));
  HCHK(r.alloc((size_t)cn * ISPMV_CHUNK_SIZE, &res, true));
  HCHK(r.alloc(n, &ord, true));
  const UIN it = ispmv_get_num_ite();
  double et = 0.0, ot = 0.0;
  HCHK(r.time(it, [&] { return ispmv_dev_int_k1(cn, d.val, d.col, d.chp, d.nmc, d.x, res, nullptr); }, no_clear,
              &et));
  HCHK(r.time(it, [&] { return ispmv_dev_order_k1(n, d.permi, res, ord, nullptr); }, no_clear, &ot));
  str_res sr = make_res("int_k1", et, ot, matK1.nnz);
  finish(fn, &sr, ord, n, ref);
  return sr;
}

ISPMV_API str_res test_int_k1p(const UIN ompNT, const str_matK1 matK1, const FPT *vec, const FPT *ref) {
  const char *fn = "test_int_k1p";
  (void)ompNT;
  const UIN cn = matK1.chunkNum, n = matK1.nrows;
  // the tail mask of the last chunk (M:1076-1086): lanes past nrows are off
  const UIN pad = cn * ISPMV_CHUNK_SIZE - n;
  const unsigned char mask = (unsigned char)(0xFFu >> (pad < 8 ? pad : 8));
  Run r;
  K1Dev d;
  FPT *res;
  HCHK(r.events());
  HCHK(upload_k1(r, matK1, vec, &d));
  HCHK(r.alloc((size_t)n + 1, &res, true));
  double et = 0.0;
  HCHK(r.time(ispmv_get_num_ite(),
              [&] { return ispmv_dev_int_k1p(mask, cn, d.val, d.col, d.chp, d.nmc, d.permi, d.x, res, nullptr); },
              no_clear, &et));
  str_res sr = make_res("int_k1p", et, 0.0, matK1.nnz);
  finish(fn, &sr, res, n, ref);
  return sr;
}

namespace {
// The AXT arrays on the device and a y of nrows entries zeroed before each run.
struct AxtDev {
  FPT *ax, *y;
  UIN *sec;
};
int upload_axt(Run &r, const str_matAXT &m, AxtDev *d) {
  int st;
  if ((st = r.up(m.ax, m.lenAX, &d->ax))) return st;
  if ((st = r.up(m.sec, m.lenSEC, &d->sec))) return st;
  return r.alloc(m.nrows, &d->y, true);
}
}  // namespace

ISPMV_API str_res test_int_axt_noc_h1(const UIN ompNT, const str_matAXT matAXT, const FPT *ref) {
  const char *fn = "test_int_axt_noc_h1";
  (void)ompNT;
  Run r;
  AxtDev d;
  HCHK(r.events());
  HCHK(upload_axt(r, matAXT, &d));
  const size_t yb = (size_t)matAXT.nrows * sizeof(FPT);
  double et = 0.0;
  HCHK(r.time(ispmv_get_num_ite(), [&] { return ispmv_dev_int_axt_noc_h1(matAXT.tileN, d.ax, d.sec, d.y, nullptr); },
              [&] { return zero(d.y, yb); }, &et));
  str_res sr = make_res("int_axt_noc_h1_hw8", et, 0.0, matAXT.nnz);
  finish(fn, &sr, d.y, matAXT.nrows, ref);
  return sr;
}

ISPMV_API str_res test_int_axt_noc(const UIN ompNT, const str_matAXT matAXT, const FPT *ref) {
  const char *fn = "test_int_axt_noc";
  (void)ompNT;
  Run r;
  AxtDev d;
  HCHK(r.events());
  HCHK(upload_axt(r, matAXT, &d));
  const size_t yb = (size_t)matAXT.nrows * sizeof(FPT);
  double et = 0.0;
  HCHK(r.time(ispmv_get_num_ite(),
              [&] { return ispmv_dev_int_axt_noc(matAXT.tileN, matAXT.tileH, d.ax, d.sec, d.y, nullptr); },
              [&] { return zero(d.y, yb); }, &et));
  char name[32];
  snprintf(name, sizeof name, "int_axt_noc_h%u_hw8", matAXT.tileH);
  str_res sr = make_res(name, et, 0.0, matAXT.nnz);
  finish(fn, &sr, d.y, matAXT.nrows, ref);
  return sr;
}

ISPMV_API str_res test_int_axt_com_h1(const UIN ompNT, const UIN bs, const str_matAXT matAXT, const FPT *ref) {
  const char *fn = "test_int_axt_com_h1";
  (void)ompNT;
  if (bs == 0) die(fn, fail(ISPMV_ERR_ARG, "test_int_axt_com_h1: bs = 0"));
  const UIN tn = matAXT.tileN, bn = (UIN)(((uint64_t)tn * ISPMV_HBRICK_SIZE + bs - 1) / bs);  // M:1580
  Run r;
  AxtDev d;
  HCHK(r.events());
  HCHK(upload_axt(r, matAXT, &d));
  const size_t yb = (size_t)matAXT.nrows * sizeof(FPT);
  double et = 0.0;
  HCHK(r.time(ispmv_get_num_ite(),
              [&] {
                return ispmv_dev_int_axt_com_h1(bn, bs, matAXT.log, matAXT.tileHW, tn, matAXT.lenAX, matAXT.lenSEC,
                                                d.ax, d.sec, d.y, nullptr);
              },
              [&] { return zero(d.y, yb); }, &et));
  char name[32];
  snprintf(name, sizeof name, "int_axt_com_h1_hw8_bs%u", bs);
  str_res sr = make_res(name, et, 0.0, matAXT.nnz);
  finish(fn, &sr, d.y, matAXT.nrows, ref);
  return sr;
}
