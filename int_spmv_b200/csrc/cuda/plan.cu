// plan.cu - plans: a format uploaded once to HBM as a value stream and a
// column-index stream plus the format's row structure, then y = A*x +
// beta*y for a fresh x on every call.
//
// Device layouts (all slot streams in the reference format's own slot
// order, x halves of `ax` dropped and replaced by the column companion):
//   CSR      val[nnz], col[nnz], row[n+1]                    (csr_vec)
//   AXC      val/col[lenAX/2] in brick order, brick row pointer brp/16
//   K1       val/col[lenVC] column-major per chunk, chp, nmc, permi
//   AXT NOC  val/col[lenAX/2] in tile order, sec cut to the used units
//   AXT COM  val/col[nnz] (packed = CSR order), a row-start bitmap (1 bit
//            per slot) and a per-segment start count instead of the
//            reference's 4-byte-per-slot descriptors, plus the compressed ->
//            real row map when some rows are empty.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "plan_kernels.cuh"

using namespace ispmv;

enum PlanFormat { F_CSR = 0, F_AXC = 1, F_K1 = 2, F_K1P = 3, F_AXT_NOC = 4, F_AXT_COM = 5 };

struct ispmv_plan_s {
  int fmt = 0;
  ispmv_plan_opts opts{};
  int device = 0;
  UIN n = 0, nnz = 0, th = 1, bs = 0, lanes = 8;
  size_t slots = 0, nunits = 0;
  UIN useg = 0;
  size_t nseg = 0;
  void *val = nullptr;  // double or float
  UIN *col = nullptr;
  UIN *rows = nullptr;  // row / brick pointer, or unit rows
  UIN *heads = nullptr, *segh = nullptr, *rowmap = nullptr, *empty = nullptr;
  size_t nempty = 0;
  UIN *chp = nullptr, *nmc = nullptr, *permi = nullptr;
  UIN chunkNum = 0;
  FPT *res = nullptr;  // K1 result in chunk order
  UIN *rec_row = nullptr;
  double *rec_sum = nullptr;
  FPT *hx = nullptr, *hy = nullptr;  // device staging of ispmv_plan_spmv_host
  std::vector<void *> owned;
  ispmv_plan_info info{};
};

namespace {

template <typename T>
int dev_upload(ispmv_plan_s *p, const T *h, size_t n, T **d) {
  void *ptr = nullptr;
  ISPMV_TRY(cudaMalloc(&ptr, (n ? n : 1) * sizeof(T)));
  p->owned.push_back(ptr);
  if (n && h) ISPMV_TRY(cudaMemcpy(ptr, h, n * sizeof(T), cudaMemcpyHostToDevice));
  *d = static_cast<T *>(ptr);
  return ISPMV_OK;
}
template <typename T>
int dev_alloc(ispmv_plan_s *p, size_t n, T **d) {
  return dev_upload<T>(p, nullptr, n, d);
}

#define TRY(expr)           \
  do {                      \
    int s__ = (expr);       \
    if (s__) return s__;    \
  } while (0)

int upload_values(ispmv_plan_s *p, const std::vector<double> &v) {
  if (p->opts.val_kind == ISPMV_VAL_F64) {
    double *d;
    TRY(dev_upload(p, v.data(), v.size(), &d));
    p->val = d;
  } else if (p->opts.val_kind == ISPMV_VAL_F32) {
    std::vector<float> f(v.size());
    for (size_t i = 0; i < v.size(); i++) f[i] = (float)v[i];
    float *d;
    TRY(dev_upload(p, f.data(), f.size(), &d));
    p->val = d;
  } else {
    return ISPMV_ERR_UNSUPPORTED;
  }
  return ISPMV_OK;
}

size_t vbytes(const ispmv_plan_s *p) { return p->opts.val_kind == ISPMV_VAL_F64 ? 8 : 4; }

void finish_info(ispmv_plan_s *p, const char *name) {
  ispmv_plan_info &i = p->info;
  i.nrows = p->n;
  i.nnz = p->nnz;
  i.slots = p->slots;
  i.format = p->fmt;
  i.val_kind = p->opts.val_kind;
  i.col_kind = p->opts.col_kind;
  i.kernel = p->opts.kernel;
  i.tile_h = p->th;
  i.bs = p->bs;
  const double bv = (double)vbytes(p), bi = 4.0;
  i.alg_bytes = (double)p->nnz * (bv + bi) + (double)p->n * 16.0 + 4.0 * ((double)p->n + 1.0);
  snprintf(i.name, sizeof i.name, "%s", name);
}

// segment sizes: about 2048 slots per warp, a multiple of 32 units
UIN pick_useg(ispmv_plan_s *p, UIN slots_per_unit) {
  UIN u = p->opts.units_per_warp;
  if (!u) u = std::max<UIN>(32u, (2048u / std::max<UIN>(1u, slots_per_unit)) & ~31u);
  u = std::max<UIN>(32u, u & ~31u);
  return u;
}

int alloc_records(ispmv_plan_s *p) {
  p->nseg = (p->nunits + p->useg - 1) / p->useg;
  TRY(dev_alloc(p, std::max<size_t>(1, 2 * p->nseg), &p->rec_row));
  TRY(dev_alloc(p, std::max<size_t>(1, 2 * p->nseg), &p->rec_sum));
  return ISPMV_OK;
}

int empty_rows(ispmv_plan_s *p, const str_matCSR *csr) {
  std::vector<UIN> e;
  for (UIN r = 0; r < csr->nrows; r++)
    if (csr->row[r + 1] == csr->row[r]) e.push_back(r);
  p->nempty = e.size();
  if (!e.empty()) TRY(dev_upload(p, e.data(), e.size(), &p->empty));
  return ISPMV_OK;
}

int check_csr(const str_matCSR *csr) {
  if (!csr || !csr->row || csr->nrows == 0) return ISPMV_ERR_ARG;
  if (csr->nnz && (!csr->col || !csr->val)) return ISPMV_ERR_ARG;
  if (csr->row[0] != 0 || csr->row[csr->nrows] != csr->nnz) return ISPMV_ERR_ARG;
  return ISPMV_OK;
}

int begin(const ispmv_plan_opts *o, ispmv_plan_s **out) {
  if (!out) return ISPMV_ERR_ARG;
  *out = nullptr;
  auto *p = new (std::nothrow) ispmv_plan_s();
  if (!p) return ISPMV_ERR_OOM;
  if (o) p->opts = *o;
  else ispmv_plan_opts_default(&p->opts);
  if (p->opts.val_kind != ISPMV_VAL_F64 && p->opts.val_kind != ISPMV_VAL_F32) {
    delete p;
    return ISPMV_ERR_UNSUPPORTED;
  }
  if (p->opts.col_kind != ISPMV_COL_U32) {
    delete p;
    return ISPMV_ERR_UNSUPPORTED;
  }
  cudaGetDevice(&p->device);
  *out = p;
  return ISPMV_OK;
}

int done(ispmv_plan_s *p, int st, ispmv_plan *out) {
  if (st != ISPMV_OK) {
    ispmv_plan_destroy(p);
    return st;
  }
  *out = p;
  return ISPMV_OK;
}

}  // namespace

ISPMV_API void ispmv_plan_opts_default(ispmv_plan_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->val_kind = ISPMV_VAL_F64;
  o->col_kind = ISPMV_COL_U32;
  o->kernel = ISPMV_KERNEL_AUTO;
}

ISPMV_API int ispmv_plan_destroy(ispmv_plan p) {
  if (!p) return ISPMV_OK;
  for (void *q : p->owned) cudaFree(q);
  delete p;
  return ISPMV_OK;
}

// ---------------------------------------------------------------- CSR --
ISPMV_API int ispmv_plan_csr(const str_matCSR *csr, const ispmv_plan_opts *o, ispmv_plan *out) {
  TRY(check_csr(csr));
  ispmv_plan_s *p;
  TRY(begin(o, &p));
  p->fmt = F_CSR;
  p->n = csr->nrows;
  p->nnz = csr->nnz;
  p->slots = csr->nnz;
  const double mean = (double)csr->nnz / csr->nrows;
  p->lanes = mean <= 2.5 ? 2 : mean <= 5 ? 4 : mean <= 12 ? 8 : mean <= 24 ? 16 : 32;
  std::vector<double> v(csr->val, csr->val + csr->nnz);
  int st = upload_values(p, v);
  if (!st) st = dev_upload(p, csr->col, csr->nnz, &p->col);
  if (!st) st = dev_upload(p, csr->row, (size_t)csr->nrows + 1, &p->rows);
  finish_info(p, "CSR");
  p->info.device_bytes = (uint64_t)csr->nnz * (vbytes(p) + 4) + 4ull * (csr->nrows + 1);
  return done(p, st, out);
}

// ---------------------------------------------------------------- AXC --
ISPMV_API int ispmv_plan_axc(const str_matCSR *csr, const str_matAXC *axc, const UIN *axi,
                             const ispmv_plan_opts *o, ispmv_plan *out) {
  TRY(check_csr(csr));
  if (!axc || !axi || !axc->ax || !axc->brp || axc->nrows != csr->nrows) return ISPMV_ERR_ARG;
  ispmv_plan_s *p;
  TRY(begin(o, &p));
  p->fmt = F_AXC;
  p->n = csr->nrows;
  p->nnz = csr->nnz;
  p->slots = axc->lenAX / 2;
  std::vector<double> v(p->slots);
  for (size_t s = 0; s < p->slots; s++) v[s] = axc->ax[(s / 8) * 16 + s % 8];
  std::vector<UIN> bptr((size_t)p->n + 1);
  for (size_t r = 0; r <= p->n; r++) bptr[r] = axc->brp[r] / 16;
  int st = upload_values(p, v);
  if (!st) st = dev_upload(p, axi, p->slots, &p->col);
  if (!st) st = dev_upload(p, bptr.data(), bptr.size(), &p->rows);
  finish_info(p, "AXC");
  p->info.device_bytes = (uint64_t)p->slots * (vbytes(p) + 4) + 4ull * (p->n + 1);
  return done(p, st, out);
}

// ----------------------------------------------------------------- K1 --
ISPMV_API int ispmv_plan_k1(const str_matCSR *csr, const str_matK1 *k1, int reorder, const ispmv_plan_opts *o,
                            ispmv_plan *out) {
  TRY(check_csr(csr));
  if (!k1 || !k1->val || !k1->col || !k1->chp || !k1->nmc || !k1->permi || k1->nrows != csr->nrows)
    return ISPMV_ERR_ARG;
  ispmv_plan_s *p;
  TRY(begin(o, &p));
  p->fmt = reorder ? F_K1P : F_K1;
  p->n = csr->nrows;
  p->nnz = csr->nnz;
  p->slots = k1->lenVC;
  p->chunkNum = k1->chunkNum;
  std::vector<double> v(k1->val, k1->val + k1->lenVC);
  int st = upload_values(p, v);
  if (!st) st = dev_upload(p, k1->col, k1->lenVC, &p->col);
  if (!st) st = dev_upload(p, k1->chp, k1->chunkNum, &p->chp);
  if (!st) st = dev_upload(p, k1->nmc, k1->chunkNum, &p->nmc);
  if (!st) st = dev_upload(p, k1->permi, (size_t)k1->chunkNum * 8, &p->permi);
  if (!st && !reorder) st = dev_alloc(p, (size_t)k1->chunkNum * 8, &p->res);
  finish_info(p, reorder ? "K1P" : "K1");
  p->info.device_bytes = (uint64_t)p->slots * (vbytes(p) + 4) + 8ull * k1->chunkNum + 32ull * k1->chunkNum;
  return done(p, st, out);
}

// ---------------------------------------------------------------- AXT --
ISPMV_API int ispmv_plan_axt(const str_matCSR *csr, const str_matAXT *axt, const UIN *axi, const ispmv_plan_opts *o,
                             ispmv_plan *out) {
  TRY(check_csr(csr));
  if (!axt || !axi || !axt->ax || !axt->sec || axt->nrows != csr->nrows) return ISPMV_ERR_ARG;
  if (axt->tileHW != 8 || axt->tileH == 0) return ISPMV_ERR_UNSUPPORTED;
  const bool com = std::strncmp(axt->mode, "COM", 3) == 0;
  const bool noc = std::strncmp(axt->mode, "NOC", 3) == 0;
  if (!com && !noc) return ISPMV_ERR_ARG;
  ispmv_plan_s *p;
  TRY(begin(o, &p));
  p->n = csr->nrows;
  p->nnz = csr->nnz;
  p->th = axt->tileH;
  int st = ISPMV_OK;
  char name[32];
  if (noc) {
    p->fmt = F_AXT_NOC;
    const UIN th = axt->tileH, grp = th == 1 ? 8 : th;
    size_t slots = 0;
    for (UIN r = 0; r < p->n; r++) slots += ((size_t)csr->rl[r] + grp - 1) / grp * grp;
    p->slots = (size_t)axt->lenAX / 2;
    p->nunits = th == 1 ? slots / 8 : slots / th;  // used tiles / tile columns
    std::vector<double> v(p->slots);
    for (size_t s = 0; s < p->slots; s++) v[s] = axt->ax[(s / 8) * 16 + s % 8];
    st = upload_values(p, v);
    if (!st) st = dev_upload(p, axi, p->slots, &p->col);
    if (!st) st = dev_upload(p, axt->sec, p->nunits, &p->rows);
    p->useg = pick_useg(p, th == 1 ? 8 : th);
    snprintf(name, sizeof name, "AXT_NOC_H%u", th);
  } else {
    if (axt->tileH != 1) { ispmv_plan_destroy(p); return ISPMV_ERR_UNSUPPORTED; }
    p->fmt = F_AXT_COM;
    p->bs = 1u << axt->log;
    p->slots = csr->nnz;
    p->nunits = csr->nnz;
    std::vector<double> v(p->slots);
    std::vector<UIN> c(p->slots);
    for (size_t s = 0; s < p->slots; s++) {
      v[s] = axt->ax[(s / 8) * 16 + s % 8];
      c[s] = axi[s];
    }
    st = upload_values(p, v);
    if (!st) st = dev_upload(p, c.data(), c.size(), &p->col);
    p->useg = pick_useg(p, 1);
    // row-start bitmap, per-segment start counts, compressed -> real rows
    const size_t nw = (p->slots + 31) / 32;
    std::vector<UIN> heads(std::max<size_t>(1, nw), 0), rowmap;
    bool any_empty = false;
    for (UIN r = 0; r < p->n; r++) {
      if (csr->row[r + 1] == csr->row[r]) { any_empty = true; continue; }
      const size_t s = csr->row[r];
      heads[s >> 5] |= 1u << (s & 31);
      rowmap.push_back(r);
    }
    const size_t nseg = (p->nunits + p->useg - 1) / p->useg;
    std::vector<UIN> segh(std::max<size_t>(1, nseg), 0);
    UIN acc = 0;
    for (size_t sg = 0, w = 0; sg < nseg; sg++) {
      const size_t wend = (sg * p->useg) >> 5;
      for (; w < wend; w++) acc += __builtin_popcount(heads[w]);
      segh[sg] = acc;
    }
    if (!st) st = dev_upload(p, heads.data(), heads.size(), &p->heads);
    if (!st) st = dev_upload(p, segh.data(), segh.size(), &p->segh);
    if (!st && any_empty) st = dev_upload(p, rowmap.data(), rowmap.size(), &p->rowmap);
    snprintf(name, sizeof name, "AXT_COM_BS%u", p->bs);
  }
  if (!st) st = empty_rows(p, csr);
  if (!st) st = alloc_records(p);
  finish_info(p, name);
  p->info.device_bytes = (uint64_t)p->slots * (vbytes(p) + 4);
  return done(p, st, out);
}

ISPMV_API int ispmv_plan_get_info(ispmv_plan p, ispmv_plan_info *info) {
  if (!p || !info) return ISPMV_ERR_ARG;
  *info = p->info;
  return ISPMV_OK;
}

// ------------------------------------------------------------ execute --
namespace {

template <typename VT>
int run(ispmv_plan_s *p, const FPT *x, FPT *y, int beta, cudaStream_t s) {
  const VT *val = static_cast<const VT *>(p->val);
  switch (p->fmt) {
    case F_CSR: {
      const size_t thr = (size_t)p->n * p->lanes;
      const unsigned g = (unsigned)((thr + pk::TPB - 1) / pk::TPB);
      switch (p->lanes) {
        case 2: pk::csr_vec<VT, 2><<<g, pk::TPB, 0, s>>>(p->n, p->rows, p->col, val, x, y, beta); break;
        case 4: pk::csr_vec<VT, 4><<<g, pk::TPB, 0, s>>>(p->n, p->rows, p->col, val, x, y, beta); break;
        case 8: pk::csr_vec<VT, 8><<<g, pk::TPB, 0, s>>>(p->n, p->rows, p->col, val, x, y, beta); break;
        case 16: pk::csr_vec<VT, 16><<<g, pk::TPB, 0, s>>>(p->n, p->rows, p->col, val, x, y, beta); break;
        default: pk::csr_vec<VT, 32><<<g, pk::TPB, 0, s>>>(p->n, p->rows, p->col, val, x, y, beta); break;
      }
      return check_launch("csr_vec");
    }
    case F_AXC: {
      const unsigned g = (unsigned)(((size_t)p->n * 8 + pk::TPB - 1) / pk::TPB);
      pk::axc_rows<VT><<<g, pk::TPB, 0, s>>>(p->n, p->rows, p->col, val, x, y, beta);
      return check_launch("axc_rows");
    }
    case F_K1:
    case F_K1P: {
      const unsigned g = (unsigned)(((size_t)p->chunkNum * 8 + pk::TPB - 1) / pk::TPB);
      if (p->fmt == F_K1P) {
        pk::k1_chunks<VT, true><<<g, pk::TPB, 0, s>>>(p->n, p->chunkNum, p->chp, p->nmc, p->permi, p->col, val, x, y,
                                                      beta);
        return check_launch("k1_chunks<scatter>");
      }
      pk::k1_chunks<VT, false><<<g, pk::TPB, 0, s>>>(p->n, p->chunkNum, p->chp, p->nmc, p->permi, p->col, val, x,
                                                     p->res, beta);
      int st = check_launch("k1_chunks");
      if (st) return st;
      pk::k1_order<<<(unsigned)((p->n + 255) / 256), 256, 0, s>>>(p->n, p->permi, p->res, y, beta);
      return check_launch("k1_order");
    }
    case F_AXT_NOC:
    case F_AXT_COM: {
      seg::Out o{y, p->rowmap, p->rec_row, p->rec_sum, beta};
      if (p->nunits) {
        const unsigned g = (unsigned)((p->nseg * 32 + pk::TPB - 1) / pk::TPB);
        if (p->fmt == F_AXT_COM) {
          pk::com_slots<VT><<<g, pk::TPB, 0, s>>>(p->nunits, p->useg, p->heads, p->segh, p->col, val, x, o);
        } else if (p->th == 1) {
          pk::noc_h1<VT><<<g, pk::TPB, 0, s>>>(p->nunits, p->useg, p->rows, p->col, val, x, o);
        } else {
          pk::noc_hn<VT><<<g, pk::TPB, 0, s>>>(p->nunits, p->th, p->useg, p->rows, p->col, val, x, o);
        }
        int st = check_launch("axt main");
        if (st) return st;
      }
      const size_t nrec = 2 * p->nseg;
      const size_t work = std::max(nrec, p->nempty);
      if (work) {
        seg::fixup<<<(unsigned)((work + 255) / 256), 256, 0, s>>>(nrec, p->rec_row, p->rec_sum, p->rowmap, p->empty,
                                                                  p->nempty, y, beta);
        return check_launch("fixup");
      }
      return ISPMV_OK;
    }
    default:
      return ISPMV_ERR_ARG;
  }
}

}  // namespace

ISPMV_API int ispmv_plan_spmv(ispmv_plan p, const FPT *x, FPT *y, int beta, void *stream) {
  if (!p || !x || !y || (beta != 0 && beta != 1)) return ISPMV_ERR_ARG;
  cudaStream_t s = as_stream(stream);
  if (p->opts.val_kind == ISPMV_VAL_F64) return run<double>(p, x, y, beta, s);
  return run<float>(p, x, y, beta, s);
}

ISPMV_API int ispmv_plan_spmv_host(ispmv_plan p, const FPT *h_x, FPT *h_y, void *stream) {
  if (!p || !h_x || !h_y) return ISPMV_ERR_ARG;
  if (!p->hx) {
    TRY(dev_alloc(p, p->n, &p->hx));
    TRY(dev_alloc(p, p->n, &p->hy));
  }
  cudaStream_t s = as_stream(stream);
  ISPMV_TRY(cudaMemcpyAsync(p->hx, h_x, (size_t)p->n * sizeof(FPT), cudaMemcpyHostToDevice, s));
  TRY(ispmv_plan_spmv(p, p->hx, p->hy, 0, stream));
  ISPMV_TRY(cudaMemcpyAsync(h_y, p->hy, (size_t)p->n * sizeof(FPT), cudaMemcpyDeviceToHost, s));
  ISPMV_TRY(cudaStreamSynchronize(s));
  return ISPMV_OK;
}

ISPMV_API int ispmv_plan_spmm(ispmv_plan p, UIN k, const FPT *X, FPT *Y, void *stream) {
  (void)p; (void)k; (void)X; (void)Y; (void)stream;
  return ISPMV_ERR_UNSUPPORTED;
}
