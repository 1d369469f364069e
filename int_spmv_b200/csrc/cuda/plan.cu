// plan.cu - plans: a format uploaded once to HBM as a value stream and a
// column-index stream plus the format's row structure, then y = A*x +
// beta*y for a fresh x on every call.
//
// Device layouts (slot streams in the reference format's own slot order; the
// x halves of `ax` are dropped and the column companion takes their place):
//   stream  CSR / AXT COM (CSR order), AXT NOC tileH=1 (tile order, rows
//           padded to 8) and AXC (brick order, rows padded to 8): val[S],
//           col[S] zero-padded to a multiple of 512 slots, a row-start bitmap
//           (1 bit per slot), per-segment start counts, and the compressed ->
//           real row map when some rows are empty.  Kernels: sss::stream_ldg,
//           sss::stream_tma; wide::stream_wide reads val/col from a
//           lane-interleaved copy (wide::il_pos) instead of slot order.
//   units   AXT NOC tileH>1 (tile columns): val/col in tile order plus the
//           reference's per-column row array (sec) cut to the used columns.
//           Kernels: pk::noc_hn, tk::nocn_tma.
//   rows    CSR row pointer (pk::csr_vec) and AXC brick pointer
//           (pk::axc_rows): the row-parallel kernels.
//   K1      val/col column-major per chunk, chp, nmc, permi (pk::k1_chunks).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_radix_sort.cuh>

#include "plan_tma.cuh"
#include "spmm.cuh"
#include "sss.cuh"
#include "tmem.cuh"
#include "wide.cuh"

using namespace ispmv;

enum PlanFormat { F_CSR = 0, F_AXC = 1, F_K1 = 2, F_K1P = 3, F_AXT_NOC = 4, F_AXT_COM = 5 };
enum PlanPath { P_STREAM = 0, P_UNITS = 1, P_ROWS = 2, P_K1 = 3 };

struct ispmv_plan_s {
  int fmt = 0;
  int path = P_STREAM;
  ispmv_plan_opts opts{};
  UIN n = 0, nnz = 0, th = 1, bs = 0, lanes = 8;
  size_t slots = 0, slots_pad = 0, nunits = 0;
  size_t seg_slots = 0, nseg = 0;
  UIN useg = 0;
  void *val = nullptr;  // double or float
  UIN *col = nullptr;
  UIN *rows = nullptr;  // row / brick pointer, or unit rows
  UIN *heads = nullptr, *segh = nullptr, *rowmap = nullptr, *empty = nullptr;
  size_t nempty = 0;
  size_t nrowmap = 0;   // entries of rowmap (0: no empty rows, no map)
  UIN *chp = nullptr, *nmc = nullptr, *permi = nullptr;
  UIN chunkNum = 0;
  FPT *res = nullptr;  // K1 result in chunk order
  UIN *rec_row = nullptr;
  double *rec_sum = nullptr;
  int *status = nullptr;
  sss::Narrow narrow{};   // D16 / LO side streams (stream path only)
  sss::XWin xw{};         // x bands staged in shared memory (variants >= 8)
  double lo_frac = 0.0;   // fraction of slots carrying a lo-word
  size_t esc_batches = 0; // D16 batches kept as u32 columns
  size_t d16_batch = 128;  // D16 slots per base column (128; 32*slots per lane for stream_wide)
  FPT *hx = nullptr, *hy = nullptr;  // device staging of ispmv_plan_spmv_host
  float *x32 = nullptr;              // FP32 copy of x (FP32-value stream_wide plans)
  cudaTextureObject_t xtex = 0;      // linear texture over x (stream_wide texture-gather variants)
  const void *xtex_src = nullptr;    // the buffer it covers
  size_t xtex_bytes = 0;
  uint32_t *tblocks = nullptr;       // the stream in TMEM-staged blocks (stream_tmem variants)
  unsigned long long *queue = nullptr;  // work-queue counter (variant ISPMV_VARIANT_QUEUE)
  cudaStream_t cap_stream = nullptr;    // private stream for graph capture
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  const FPT *g_x = nullptr;
  FPT *g_y = nullptr;
  int g_beta = -1;
  UIN *mm_row = nullptr;             // SpMM records (allocated on first use)
  double *mm_sum = nullptr;
  size_t mm_cap = 0;                 // doubles in mm_sum
  size_t mm_rows_cap = 0;            // entries of mm_row
  UIN k1_long = 0;                   // K1: leading chunks run a warp each
  std::vector<void *> owned;
  ispmv_plan_info info{};
  std::vector<cudaEvent_t> tev;      // kernel timing: event pairs around the main kernel (a ring)
  size_t tcap = 0;                   // pairs in the ring (0: timing off)
  size_t tcount = 0;                 // pairs recorded since the last read
  bool capturing = false;            // inside graph capture: no timing events
  const char *kname = "";            // main kernel of the latest product (a static string)
};

namespace {

constexpr size_t SS = sss::SS;      // slots per staged stage; streams pad to it
constexpr size_t SEG_SLOTS = 2048;  // default slots per warp segment
constexpr UIN K1_LONG = 64;         // K1 chunks of at least this many columns run a warp each

#define TRY(expr)        \
  do {                   \
    int s__ = (expr);    \
    if (s__) return s__; \
  } while (0)

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

size_t vbytes(const ispmv_plan_s *p) { return p->opts.val_kind == ISPMV_VAL_F64 ? 8 : 4; }

// The reduced-byte side streams exist only on the slot-stream path.
bool narrow_kinds(const ispmv_plan_s *p) {
  return p->opts.val_kind == ISPMV_VAL_F32_LO16 || p->opts.col_kind == ISPMV_COL_D16;
}

uint16_t to_bf16(float f) {  // round to nearest even
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

int upload_values(ispmv_plan_s *p, const std::vector<double> &v) {
  if (p->opts.val_kind == ISPMV_VAL_F64) {
    double *d;
    TRY(dev_upload(p, v.data(), v.size(), &d));
    p->val = d;
    return ISPMV_OK;
  }
  // FP32 (and the hi part of FP32 + lo-word)
  std::vector<float> f(v.size());
  for (size_t i = 0; i < v.size(); i++) f[i] = (float)v[i];
  float *d;
  TRY(dev_upload(p, f.data(), f.size(), &d));
  p->val = d;
  return ISPMV_OK;
}

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
  // b_val: 8 | 4 | 4 + 2*(lo-word fraction); b_idx: 4 | 2 + 4*(batch bases + escaped columns)/nnz
  double bv = (double)vbytes(p), bi = 4.0;
  if (p->opts.val_kind == ISPMV_VAL_F32_LO16) bv = 4.0 + 2.0 * p->lo_frac;
  if (p->opts.col_kind == ISPMV_COL_D16 && p->slots_pad) {
    const double B = (double)p->d16_batch, batches = (double)(p->slots_pad / p->d16_batch);
    bi = 2.0 + (4.0 * batches + B * 4.0 * (double)p->esc_batches) / std::max(1.0, (double)p->nnz);
  }
  i.alg_bytes = (double)p->nnz * (bv + bi) + (double)p->n * 16.0 + 4.0 * ((double)p->n + 1.0);
  snprintf(i.name, sizeof i.name, "%s", name);
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
  if (p->opts.val_kind < ISPMV_VAL_F64 || p->opts.val_kind > ISPMV_VAL_F32_LO16 || p->opts.col_kind < ISPMV_COL_U32 ||
      p->opts.col_kind > ISPMV_COL_D16 || p->opts.kernel < 0 || p->opts.kernel > ISPMV_KERNEL_WIDE ||
      (p->opts.spmm_kernel != ISPMV_KERNEL_AUTO && p->opts.spmm_kernel != ISPMV_KERNEL_LDG &&
       p->opts.spmm_kernel != ISPMV_KERNEL_WIDE)) {
    delete p;
    return ISPMV_ERR_UNSUPPORTED;
  }
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

int empty_rows(ispmv_plan_s *p, const str_matCSR *csr) {
  std::vector<UIN> e;
  for (UIN r = 0; r < csr->nrows; r++)
    if (csr->row[r + 1] == csr->row[r]) e.push_back(r);
  p->nempty = e.size();
  if (!e.empty()) TRY(dev_upload(p, e.data(), e.size(), &p->empty));
  return ISPMV_OK;
}

int alloc_records(ispmv_plan_s *p) {
  TRY(dev_alloc(p, std::max<size_t>(1, 2 * p->nseg), &p->rec_row));
  TRY(dev_alloc(p, std::max<size_t>(1, 2 * p->nseg), &p->rec_sum));
  TRY(dev_alloc(p, 1, &p->status));
  ISPMV_TRY(cudaMemset(p->status, 0, sizeof(int)));
  TRY(dev_alloc(p, 1, &p->queue));
  return ISPMV_OK;
}

size_t seg_slots_of(const ispmv_plan_s *p, size_t upu) {
  if (p->opts.units_per_warp <= 0) return SEG_SLOTS;
  return std::max(SS, ((size_t)p->opts.units_per_warp * upu + SS - 1) / SS * SS);
}

// stream_wide variants, numbered as measured (numbers not listed here were
// measured and retired: x bands in shared memory, per-warp row buffers,
// other segment sizes, stage counts and window sizes):
// slots per lane, per-CTA x window (cap doubles), segment slots, CTAs per SM
// the registers are sized for (plain loads), and for the staged form (tma)
// the stages per warp and warps per CTA.
struct WideCfg {
  int spl; UIN cap; size_t seg; int minb; bool tma; int stages; int warps; bool tex = false;
  bool tmem = false;  // stream staged through tensor memory (stream_tmem); stages = TMEM stages,
                      // warps = consumer warps per CTA (4 per column half)
  bool stg = false;   // one x window per CTA (cap doubles), chosen at plan time, copied by one bulk copy
  bool pfc = false;   // the next batch's columns loaded one batch ahead
  bool ok = true;     // a variant this build runs
};
constexpr int WIDE_WARPS = 8;
WideCfg wide_variant(int v) {
  switch (v) {
    case 0: return {16, 0, 4096, 3, false, 0, 8};
    case 4: return {8, 0, 2048, 4, false, 0, 8};
    case 8: return {16, 0, 8192, 3, false, 0, 8};
    case 9: return {16, 0, 2048, 3, false, 0, 8};
    case 11: return {16, 0, 4096, 0, true, 2, 4};                            // bulk-copy staged stream
    case 16: return {8, 0, 2048, 4, false, 0, 8, true};                      // texture gathers
    case 18: return {8, 0, 8192, 0, false, 4, 4, false, true};               // TMEM-staged stream
    case 19: return {16, 0, 8192, 0, false, 2, 4, false, true};
    case 20: return {8, 0, 8192, 0, false, 2, 8, false, true};
    case 21: return {16, 0, 8192, 0, false, 2, 8, false, true};
    case 26: return {8, 3584, 1536, 4, false, 0, 8, false, false, true};     // per-CTA x window, one bulk copy
    case 32: return {8, 0, 2048, 4, false, 0, 8, false, false, false, true}; // next batch's columns ahead
    default: {
      WideCfg c{16, 0, 4096, 3, false, 0, 8};
      c.ok = false;
      return c;
    }
  }
}

// Fraction of a deterministic sample of the nonzeros whose column lies
// far from the diagonal (|c - r| > 1536, outside a 3072-column window) with
// no column of the next row within 16 of c + 1: gathers with no locality
// between neighbouring rows, which the L1 cache cannot share between the
// lanes of a warp (uniformly scattered columns; not the fixed far offsets
// of a stencil).  Such matrices gain from the staged per-CTA windows.
double random_far_fraction(const str_matCSR *csr) {
  const size_t nnz = csr->nnz, S = std::min<size_t>(nnz, 1u << 16);
  if (!S) return 0.0;
  const double stride = (double)nnz / (double)S;
  size_t far = 0;
  for (size_t i = 0, r = 0; i < S; i++) {
    const size_t j = (size_t)(i * stride);
    while (r < csr->nrows && csr->row[r + 1] <= j) r++;
    if (r >= csr->nrows) break;  // a row pointer that does not cover nnz
    const long long c = csr->col[j];
    if (std::llabs(c - (long long)r) <= 1536) continue;
    bool near_next = false;
    if (r + 1 < csr->nrows)
      for (UIN k = csr->row[r + 1]; k < csr->row[r + 2] && !near_next; k++)
        near_next = std::llabs((long long)csr->col[k] - c - 1) <= 16;
    far += !near_next;
  }
  return (double)far / (double)S;
}

// AUTO on a slot-stream plan: the lane-interleaved kernel (stream_wide) and
// its variant.  8 slots per lane for rows of fewer than 16 nonzeros on
// average, with per-CTA x windows where the columns are scattered (FP64
// values) or the next batch's columns loaded ahead (FP32 values, whose
// kernel has the registers for it); else 16 slots per lane, bulk-copy staged
// for FP64 values with u32 columns that are not scattered (measured fastest
// there), plain loads for scattered columns and for the FP32, lo-word and
// 16-bit-delta forms (FP32 values: 8192-slot segments).  An explicit variant
// is kept.
int auto_variant(const ispmv_plan_s *p, bool long_rows, bool scattered) {
  const bool plain = p->opts.val_kind == ISPMV_VAL_F64 && p->opts.col_kind == ISPMV_COL_U32;
  const bool f32 = p->opts.val_kind == ISPMV_VAL_F32;
  if (!long_rows) return scattered && !narrow_kinds(p) ? (f32 ? 32 : 26) : 4;
  if (plain && !scattered) return 11;
  return f32 ? 8 : 0;  // FP32 values: 8192-slot segments (measured 3% faster on the 27-point stencil)
}
void auto_wide(ispmv_plan_s *p, const str_matCSR *csr) {
  p->opts.kernel = ISPMV_KERNEL_WIDE;
  if (p->opts.variant != 0) return;
  p->opts.variant = auto_variant(p, (double)csr->nnz >= 16.0 * (double)p->n, random_far_fraction(csr) >= 0.05);
}

// The per-CTA x windows of the staged stream_wide variants: CTA t walks
// slots [t*T, (t+1)*T), T = WIDE_WARPS*seg_slots; its window is the
// cap-long interval of x holding the most of those slots' columns (padding
// slots excluded), centred on them, clamped to x and started at an even
// column, so the bulk copy starts on a 16-byte boundary and moves a
// multiple of 16 bytes, all inside x[0, n rounded down to even).  Columns
// outside a CTA's window are gathered from x.
int stage_windows(ispmv_plan_s *p, const std::vector<double> &v, const std::vector<UIN> &c) {
  const UIN W = wide_variant(p->opts.variant).cap & ~1u, ne = p->n & ~1u;
  const size_t T = (size_t)WIDE_WARPS * p->seg_slots, nt = std::max<size_t>(1, (p->nseg + WIDE_WARPS - 1) / WIDE_WARPS);
  std::vector<UIN> lo(nt, 0), len(nt, 0);
#pragma omp parallel for schedule(dynamic, 16)
  for (long long t = 0; t < (long long)nt; t++) {
    if (ne <= W) {  // all of x (but an odd last element) fits
      len[t] = ne;
      continue;
    }
    const size_t a = (size_t)t * T, e = std::min(p->slots, a + T);
    std::vector<UIN> cs;
    cs.reserve(T);
    for (size_t q = a; q < e; q++)
      if (v[q] != 0.0) cs.push_back(c[q]);
    long long l = 0;
    if (!cs.empty()) {
      std::sort(cs.begin(), cs.end());
      size_t best = 0, ba = 0, bb = 1;
      for (size_t i = 0, j = 0; i < cs.size(); i++) {  // [cs[i], cs[i] + W - 1)
        if (j < i) j = i;
        while (j < cs.size() && cs[j] - cs[i] < W - 1) j++;
        if (j - i > best) { best = j - i; ba = i; bb = j; }
      }
      const long long span = (long long)cs[bb - 1] - (long long)cs[ba] + 1;
      l = (long long)cs[ba] - ((long long)W - span) / 2;
    }
    l = std::max(0LL, std::min(l, (long long)(ne - W)));
    lo[t] = (UIN)l & ~1u;
    len[t] = W;
  }
  UIN *dlo, *dlen;
  TRY(dev_upload(p, lo.data(), lo.size(), &dlo));
  TRY(dev_upload(p, len.data(), len.size(), &dlen));
  p->xw.tlo = dlo;
  p->xw.tlen = dlen;
  p->xw.cap = W;
  p->xw.nwin = 1;
  p->xw.n = p->n;
  return ISPMV_OK;
}

// The stream path: `v`/`c` the slot streams (length p->slots), `start[r]`
// the first slot of row r (rows with no slot are skipped).
int setup_stream(ispmv_plan_s *p, const str_matCSR *csr, std::vector<double> &v, std::vector<UIN> &c,
                 const std::vector<size_t> &start) {
  p->path = P_STREAM;
  p->slots_pad = std::max(SS, (p->slots + SS - 1) / SS * SS);
  if (p->opts.kernel == ISPMV_KERNEL_WIDE && wide_variant(p->opts.variant).tmem) {
    // whole CTAs: every consumer warp of stream_tmem walks a full segment
    const size_t unit = (size_t)wide_variant(p->opts.variant).warps * wide_variant(p->opts.variant).seg;
    p->slots_pad = std::max(unit, (p->slots + unit - 1) / unit * unit);
  }
  v.resize(p->slots_pad, 0.0);
  c.resize(p->slots_pad, 0);
  std::vector<UIN> heads(p->slots_pad / 32, 0), rowmap;
  bool any_empty = false;
  for (UIN r = 0; r < p->n; r++) {
    if (csr->row[r + 1] == csr->row[r]) {
      any_empty = true;
      continue;
    }
    const size_t q = start[r];
    heads[q >> 5] |= 1u << (q & 31);
    rowmap.push_back(r);
  }
  const bool wide = p->opts.kernel == ISPMV_KERNEL_WIDE;
  size_t wide_seg = 0;
  if (wide) {
    const WideCfg wc = wide_variant(p->opts.variant);
    const bool lo16 = p->opts.val_kind == ISPMV_VAL_F32_LO16;
    if (!wc.ok) return fail(ISPMV_ERR_UNSUPPORTED, "stream_wide: no such variant");
    if ((narrow_kinds(p) && (wc.tma || wc.tmem || wc.stg || wc.pfc)) || (lo16 && wc.tex))
      return fail(ISPMV_ERR_UNSUPPORTED,
                  "stream_wide: 16-bit column deltas and BF16 lo-words on the plain-load variants "
                  "(lo-words: not the texture-gather variants)");
    wide_seg = wc.seg;
  }
  p->seg_slots = seg_slots_of(p, 1);
  if (wide && (p->opts.units_per_warp <= 0 || wide_variant(p->opts.variant).tmem)) p->seg_slots = wide_seg;
  if (wide && p->seg_slots % SS) p->seg_slots = (p->seg_slots + SS - 1) / SS * SS;
  p->nseg = (p->slots_pad + p->seg_slots - 1) / p->seg_slots;
  std::vector<UIN> segh(std::max<size_t>(1, p->nseg), 0);
  UIN acc = 0;
  for (size_t sg = 0, w = 0; sg < p->nseg; sg++) {
    const size_t wend = std::min(heads.size(), (sg * p->seg_slots) >> 5);
    for (; w < wend; w++) acc += __builtin_popcount(heads[w]);
    segh[sg] = acc;
  }
  if (wide && wide_variant(p->opts.variant).tmem) {
    // TMEM-staged blocks: block j of CTA c holds batch j of segments
    // nw*c..nw*c+nw-1, one half-block per 4 of them; in half-block h,
    // lane-row r = 32q + l (segment nw*c + 4h + q, lane l) with its SPL values
    // then its SPL columns, in the copy's canonical layout (tmemk::blk_word)
    const unsigned spl = (unsigned)wide_variant(p->opts.variant).spl, BT = 32u * spl;
    const unsigned nw = (unsigned)wide_variant(p->opts.variant).warps;  // 4 per column half
    const bool f64 = p->opts.val_kind == ISPMV_VAL_F64;
    const unsigned vw = f64 ? 2u : 1u, W = vw * spl + spl, BW = W / 8u * 1024u;  // words per half-block
    const size_t nbat = p->seg_slots / BT, nctas = p->nseg / nw;
    std::vector<uint32_t> blk(nctas * nbat * BW * (nw / 4u), 0u);
    for (size_t cta = 0; cta < nctas; cta++)
      for (size_t j = 0; j < nbat; j++)
        for (unsigned w = 0; w < nw; w++) {
          uint32_t *B = blk.data() + ((cta * nbat + j) * (nw / 4u) + w / 4u) * BW;
          const unsigned q = w % 4u;
          for (unsigned l = 0; l < 32u; l++)
            for (unsigned k = 0; k < spl; k++) {
              const size_t sl = (cta * nw + w) * p->seg_slots + j * BT + (size_t)spl * l + k;
              const unsigned r = 32u * q + l;
              if (f64) {
                uint64_t u;
                std::memcpy(&u, &v[sl], 8);
                B[tmemk::blk_word(r, 2u * k)] = (uint32_t)u;
                B[tmemk::blk_word(r, 2u * k + 1u)] = (uint32_t)(u >> 32);
              } else {
                const float f = (float)v[sl];
                std::memcpy(&B[tmemk::blk_word(r, k)], &f, 4);
              }
              B[tmemk::blk_word(r, vw * spl + k)] = c[sl];
            }
      }
    TRY(dev_upload(p, blk.data(), blk.size(), &p->tblocks));
  } else if (wide) {
    // the lane-interleaved copy: batches of 32*spl slots, one 16-byte vector per lane and step
    const unsigned spl = (unsigned)wide_variant(p->opts.variant).spl;
    std::vector<double> vi(p->slots_pad);
    std::vector<UIN> ci(p->slots_pad);
    const unsigned vv = p->opts.val_kind == ISPMV_VAL_F64 ? 2u : 4u;
    for (size_t q = 0; q < p->slots_pad; q++) {
      vi[wide::il_pos(q, spl, vv)] = v[q];
      ci[wide::il_pos(q, spl, 4u)] = c[q];
    }
    TRY(upload_values(p, vi));
    if (p->opts.col_kind == ISPMV_COL_U32) {
      TRY(dev_upload(p, ci.data(), ci.size(), &p->col));
    } else {
      // per batch of 32*spl slots: base = the smallest column among nonzero
      // values, deltas to it in 16 bits (lane-interleaved, 8 per vector), or
      // the batch's interleaved u32 columns when the span is wider
      const size_t BT = 32u * spl, nb = p->slots_pad / BT;
      p->d16_batch = BT;
      std::vector<UIN> cmeta(nb), esc;
      std::vector<uint16_t> c16(p->slots_pad, 0);
      for (size_t b = 0; b < nb; b++) {
        UIN lo = 0xFFFFFFFFu, hi = 0;
        for (size_t q = b * BT; q < b * BT + BT; q++)
          if (v[q] != 0.0) { lo = std::min(lo, c[q]); hi = std::max(hi, c[q]); }
        if (lo == 0xFFFFFFFFu) lo = hi = 0;
        if (hi - lo <= 0xFFFFu && lo < sss::ESCAPE) {
          cmeta[b] = lo;
          for (size_t q = b * BT; q < b * BT + BT; q++)
            c16[wide::il_pos(q, spl, 8u)] = v[q] != 0.0 ? (uint16_t)(c[q] - lo) : 0;
        } else {
          cmeta[b] = sss::ESCAPE | (UIN)p->esc_batches++;
          esc.insert(esc.end(), ci.begin() + b * BT, ci.begin() + b * BT + BT);  // interleaved already
        }
      }
      uint16_t *d16; UIN *dm, *de;
      TRY(dev_upload(p, c16.data(), c16.size(), &d16));
      TRY(dev_upload(p, cmeta.data(), cmeta.size(), &dm));
      TRY(dev_upload(p, esc.data(), esc.size(), &de));
      p->narrow.col16 = d16; p->narrow.cmeta = dm; p->narrow.esc = de;
    }
  } else {
    TRY(upload_values(p, v));
    if (p->opts.col_kind == ISPMV_COL_U32) TRY(dev_upload(p, c.data(), c.size(), &p->col));
  }
  if (p->opts.col_kind == ISPMV_COL_D16 && !wide) {
    // per 128-slot batch: base = the smallest column among nonzero values;
    // deltas to it in 16 bits, or the batch's u32 columns when the span is wider
    const size_t nb = p->slots_pad / 128;
    std::vector<UIN> cmeta(nb), esc;
    std::vector<uint16_t> c16(p->slots_pad, 0);
    for (size_t b = 0; b < nb; b++) {
      UIN lo = 0xFFFFFFFFu, hi = 0;
      for (size_t q = b * 128; q < b * 128 + 128; q++)
        if (v[q] != 0.0) { lo = std::min(lo, c[q]); hi = std::max(hi, c[q]); }
      if (lo == 0xFFFFFFFFu) lo = hi = 0;
      if (hi - lo <= 0xFFFFu && lo < sss::ESCAPE) {
        cmeta[b] = lo;
        for (size_t q = b * 128; q < b * 128 + 128; q++) c16[q] = v[q] != 0.0 ? (uint16_t)(c[q] - lo) : 0;
      } else {
        cmeta[b] = sss::ESCAPE | (UIN)p->esc_batches++;
        esc.insert(esc.end(), c.begin() + b * 128, c.begin() + b * 128 + 128);
      }
    }
    uint16_t *d16; UIN *dm, *de;
    TRY(dev_upload(p, c16.data(), c16.size(), &d16));
    TRY(dev_upload(p, cmeta.data(), cmeta.size(), &dm));
    TRY(dev_upload(p, esc.data(), esc.size(), &de));
    p->narrow.col16 = d16; p->narrow.cmeta = dm; p->narrow.esc = de;
  }
  if (p->opts.val_kind == ISPMV_VAL_F32_LO16) {
    // rows whose FP32 rounding error, relative to their row sum, exceeds
    // lo_tol get a BF16 residual; it is stored for every segment they touch
    const double tol = p->opts.lo_tol > 0 ? p->opts.lo_tol : 1e-6;
    std::vector<char> segflag(p->nseg, 0);
    for (UIN r = 0; r < p->n; r++) {
      double err = 0.0, sum = 0.0;
      for (UIN j = csr->row[r]; j < csr->row[r + 1]; j++) {
        err += std::fabs(csr->val[j] - (double)(float)csr->val[j]);
        sum += csr->val[j];
      }
      if (csr->row[r + 1] == csr->row[r] || err <= tol * std::fabs(sum)) continue;
      const size_t a = start[r], e = start[r] + (csr->row[r + 1] - csr->row[r]);
      for (size_t sg = a / p->seg_slots; sg <= (e - 1) / p->seg_slots && sg < p->nseg; sg++) segflag[sg] = 1;
    }
    // a flagged segment's residuals in slot order, or lane-interleaved like
    // the 16-bit deltas (8 per vector) for the lane-interleaved kernel; its
    // slot count is a multiple of the batch, so batches stay whole
    const unsigned ilspl = wide ? (unsigned)wide_variant(p->opts.variant).spl : 0u;
    std::vector<UIN> off(p->nseg, NO_ROW);
    std::vector<uint16_t> lo;
    for (size_t sg = 0; sg < p->nseg; sg++) {
      if (!segflag[sg]) continue;
      const size_t base = lo.size();
      off[sg] = (UIN)base;
      const size_t a = sg * p->seg_slots, e = std::min(p->slots_pad, a + p->seg_slots);
      lo.resize(base + (e - a));
      for (size_t q = a; q < e; q++)
        lo[base + (ilspl ? wide::il_pos(q - a, ilspl, 8u) : q - a)] = to_bf16((float)(v[q] - (double)(float)v[q]));
    }
    p->lo_frac = p->slots ? (double)lo.size() / (double)p->slots_pad : 0.0;
    uint16_t *dl; UIN *dof;
    TRY(dev_upload(p, lo.data(), lo.size(), &dl));
    TRY(dev_upload(p, off.data(), off.size(), &dof));
    p->narrow.lo16 = dl; p->narrow.lo_off = dof;
  }
  TRY(dev_upload(p, heads.data(), heads.size(), &p->heads));
  TRY(dev_upload(p, segh.data(), segh.size(), &p->segh));
  if (any_empty) TRY(dev_upload(p, rowmap.data(), rowmap.size(), &p->rowmap));
  p->nrowmap = any_empty ? rowmap.size() : 0;
  const bool stg = wide && wide_variant(p->opts.variant).stg;
  if (stg) TRY(stage_windows(p, v, c));
  TRY(empty_rows(p, csr));
  TRY(alloc_records(p));
  if (stg) p->xw.status = p->status;
  p->info.device_bytes = (uint64_t)(stg ? 8 * ((p->nseg + WIDE_WARPS - 1) / WIDE_WARPS) : 0) +
                         (uint64_t)p->slots_pad * vbytes(p) + p->slots_pad / 8 +
                         (p->opts.col_kind == ISPMV_COL_D16 ? p->slots_pad * 2 + p->slots_pad / p->d16_batch * 4 +
                                                                 p->esc_batches * p->d16_batch * 4
                                                           : p->slots_pad * 4) +
                         (uint64_t)(p->lo_frac * (double)p->slots_pad * 2.0);
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
  for (cudaEvent_t e : p->tev) cudaEventDestroy(e);
  if (p->xtex) cudaDestroyTextureObject(p->xtex);
  if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->cap_stream) cudaStreamDestroy(p->cap_stream);
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
  int st = ISPMV_OK;
  if (p->opts.kernel == ISPMV_KERNEL_AUTO) auto_wide(p, csr);  // the CSR-order slot stream
  if (p->opts.kernel == ISPMV_KERNEL_ROWS) {
    // the naive CSR product on the GPU: L lanes per row
    if (narrow_kinds(p)) { ispmv_plan_destroy(p); return ISPMV_ERR_UNSUPPORTED; }
    p->opts.kernel = ISPMV_KERNEL_ROWS;
    p->path = P_ROWS;
    const double mean = (double)csr->nnz / csr->nrows;
    p->lanes = mean <= 2.5 ? 2 : mean <= 5 ? 4 : mean <= 12 ? 8 : mean <= 24 ? 16 : 32;
    std::vector<double> v(csr->val, csr->val + csr->nnz);
    st = upload_values(p, v);
    if (!st) st = dev_upload(p, csr->col, csr->nnz, &p->col);
    if (!st) st = dev_upload(p, csr->row, (size_t)csr->nrows + 1, &p->rows);
    p->info.device_bytes = (uint64_t)csr->nnz * (vbytes(p) + 4) + 4ull * (csr->nrows + 1);
  } else {
    std::vector<double> v(csr->val, csr->val + csr->nnz);
    std::vector<UIN> c(csr->col, csr->col + csr->nnz);
    std::vector<size_t> start(csr->row, csr->row + csr->nrows);
    st = setup_stream(p, csr, v, c, start);
  }
  finish_info(p, "CSR");
  return done(p, st, out);
}

// ------------------------------------------ plans from a device CSR --
// The CSR-order slot stream (the compacted AXT's stream) built on the GPU
// from d_row / d_col / d_val, with the arrays setup_stream builds on the host
// for a lane-interleaved plan: values and columns interleaved per batch of
// 32*spl slots (wide::il_pos), zero padding to the stream length, the
// row-start bitmap, per-segment start counts, the compressed -> real row map
// (when rows are empty) and the empty-row list.  Row starts are set with
// atomicOr, so the bitmap does not depend on the order of the writes.
namespace {

// *bad = 1 if the row pointer decreases, row[0] != 0, row[n] != nnz, or a
// column is >= n.  Only reads row[0..n] and col[0..nnz).
__global__ void dcsr_check(UIN n, UIN nnz, const UIN *__restrict__ row, const UIN *__restrict__ col,
                           int *__restrict__ bad) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x, stride = (size_t)gridDim.x * blockDim.x;
  for (size_t r = i; r < n; r += stride)
    if (row[r + 1] < row[r]) *bad = 1;
  for (size_t j = i; j < nnz; j += stride)
    if (col[j] >= n) *bad = 1;
  if (i == 0 && (row[0] != 0 || row[n] != nnz)) *bad = 1;
}

// flag[r] = 1 for a row with elements; flag[n] = 0, so the exclusive prefix
// at n is the count of non-empty rows.
__global__ void dcsr_flags(UIN n, const UIN *__restrict__ row, UIN *__restrict__ flag) {
  const size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r <= n) flag[r] = r < n && row[r + 1] > row[r] ? 1u : 0u;
}

// Row-start bits, the compressed -> real map and the empty-row list from the
// prefix `pos` of the non-empty flags.
__global__ void dcsr_rows(UIN n, const UIN *__restrict__ row, const UIN *__restrict__ pos, UIN *__restrict__ heads,
                          UIN *__restrict__ rowmap, UIN *__restrict__ empty) {
  const size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const UIN a = row[r];
  if (row[r + 1] > a) {
    atomicOr(&heads[a >> 5], 1u << (a & 31u));
    if (rowmap) rowmap[pos[r]] = (UIN)r;
  } else if (empty) {
    empty[r - pos[r]] = (UIN)r;
  }
}

// segh[g] = row starts at slots below g*seg: the non-empty rows r with
// row[r] < g*seg, i.e. pos[first r with row[r] >= g*seg].
__global__ void dcsr_segh(size_t nseg, size_t seg, UIN n, const UIN *__restrict__ row, const UIN *__restrict__ pos,
                          UIN *__restrict__ segh) {
  const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nseg) return;
  const uint64_t S = (uint64_t)g * seg;
  UIN lo = 0, hi = n;  // first r in [0, n) with row[r] >= S, else n
  while (lo < hi) {
    const UIN mid = lo + (hi - lo) / 2;
    if ((uint64_t)row[mid] < S) lo = mid + 1;
    else hi = mid;
  }
  segh[g] = pos[lo];
}

// The lane-interleaved value and column copies, zero beyond nnz.
template <typename VT>
__global__ void dcsr_interleave(size_t nnz, size_t spad, unsigned spl, const UIN *__restrict__ col,
                                const FPT *__restrict__ val, VT *__restrict__ vi, UIN *__restrict__ ci) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < spad; q += stride) {
    const bool in = q < nnz;
    vi[wide::il_pos(q, spl, 16u / (unsigned)sizeof(VT))] = (VT)(in ? val[q] : 0.0);
    ci[wide::il_pos(q, spl, 4u)] = in ? col[q] : 0u;
  }
}

struct DevTmp {  // builder scratch, freed on every exit
  std::vector<void *> v;
  ~DevTmp() {
    for (void *q : v) cudaFree(q);
  }
  template <typename T>
  int alloc(size_t n, T **d) {
    void *q = nullptr;
    ISPMV_TRY(cudaMalloc(&q, (n ? n : 1) * sizeof(T)));
    v.push_back(q);
    *d = static_cast<T *>(q);
    return ISPMV_OK;
  }
};

// random_far_fraction on a device CSR: the same sample (nonzero
// j = (size_t)(i * stride)), its row by binary search (the r with
// row[r] <= j < row[r+1]), the same test; *far counts the hits.
__global__ void dcsr_far(size_t S, double stride, UIN n, const UIN *__restrict__ row, const UIN *__restrict__ col,
                         unsigned long long *__restrict__ far) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S) return;
  const size_t j = (size_t)(i * stride);
  UIN a = 1, b = n;  // first k in [1, n] with row[k] > j (row[n] = nnz > j)
  while (a < b) {
    const UIN m = a + (b - a) / 2;
    if (row[m] > j) b = m;
    else a = m + 1;
  }
  const size_t r = a - 1;
  const long long c = col[j];
  if (llabs(c - (long long)r) <= 1536) return;
  bool near_next = false;
  if (r + 1 < n)
    for (UIN k = row[r + 1]; k < row[r + 2] && !near_next; k++) near_next = llabs((long long)col[k] - c - 1) <= 16;
  if (!near_next) atomicAdd(far, 1ull);
}

// Window keys: the column of every nonzero value, ~0 for a zero value
// (sorted last, left out of the window choice as on the host).
__global__ void dcsr_win_keys(size_t nnz, const UIN *__restrict__ col, const FPT *__restrict__ val,
                              UIN *__restrict__ keys) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += stride)
    keys[q] = val[q] != 0.0 ? col[q] : 0xFFFFFFFFu;
}

__global__ void dcsr_win_offsets(size_t nt, size_t T, size_t nnz, int *__restrict__ off) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t <= nt) off[t] = (int)std::min(t * T, nnz);
}

// One CTA per plan CTA tile: stage_windows' choice from the tile's sorted
// keys - the first i with the most keys in [cs[i], cs[i] + W - 1), the
// interval centred on them, clamped to [0, ne - W], started at an even column.
__global__ void __launch_bounds__(256) dcsr_windows(size_t nt, const int *__restrict__ off,
                                                    const UIN *__restrict__ keys, UIN W, UIN ne,
                                                    UIN *__restrict__ tlo, UIN *__restrict__ tlen) {
  __shared__ UIN sb[8], si[8], sj[8];
  const size_t t = blockIdx.x;
  if (t >= nt) return;
  if (ne <= W) {
    if (threadIdx.x == 0) {
      tlo[t] = 0;
      tlen[t] = ne;
    }
    return;
  }
  const UIN *cs = keys + off[t];
  const UIN all = (UIN)(off[t + 1] - off[t]);
  UIN a = 0, b = all;  // m: keys below the sentinel
  while (a < b) {
    const UIN mid = a + (b - a) / 2;
    if (cs[mid] == 0xFFFFFFFFu) b = mid;
    else a = mid + 1;
  }
  const UIN m = a;
  UIN best = 0, bi = 0xFFFFFFFFu, bj = 0;
  for (UIN i = threadIdx.x; i < m; i += blockDim.x) {
    const uint64_t lim = (uint64_t)cs[i] + (W - 1);
    UIN lo = i, hi = m;  // first j in [i, m) with cs[j] >= lim
    while (lo < hi) {
      const UIN mid = lo + (hi - lo) / 2;
      if ((uint64_t)cs[mid] < lim) lo = mid + 1;
      else hi = mid;
    }
    if (lo - i > best) {
      best = lo - i;
      bi = i;
      bj = lo;
    }
  }
  // the largest count, the smallest i among equal counts
  for (int d = 16; d > 0; d >>= 1) {
    const UIN ob = __shfl_down_sync(FULL, best, d), oi = __shfl_down_sync(FULL, bi, d),
              oj = __shfl_down_sync(FULL, bj, d);
    if (ob > best || (ob == best && oi < bi)) {
      best = ob;
      bi = oi;
      bj = oj;
    }
  }
  const unsigned w = threadIdx.x >> 5;
  if ((threadIdx.x & 31u) == 0) {
    sb[w] = best;
    si[w] = bi;
    sj[w] = bj;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (unsigned k = 1; k < blockDim.x / 32; k++)
      if (sb[k] > best || (sb[k] == best && si[k] < bi)) {
        best = sb[k];
        bi = si[k];
        bj = sj[k];
      }
    long long l = 0;
    if (m > 0) {
      const long long span = (long long)cs[bj - 1] - (long long)cs[bi] + 1;
      l = (long long)cs[bi] - ((long long)W - span) / 2;
    }
    l = l < 0 ? 0 : l;
    l = l > (long long)(ne - W) ? (long long)(ne - W) : l;
    tlo[t] = (UIN)l & ~1u;
    tlen[t] = W;
  }
}

int dev_csr_stream(ispmv_plan_s *p, UIN n, UIN nnz, const UIN *row, const UIN *col, const FPT *val, cudaStream_t s) {
  if (p->opts.kernel != ISPMV_KERNEL_AUTO && p->opts.kernel != ISPMV_KERNEL_WIDE)
    return fail(ISPMV_ERR_UNSUPPORTED, "plan from a device CSR: the lane-interleaved kernel");
  if (p->opts.val_kind == ISPMV_VAL_F32_LO16 || p->opts.col_kind != ISPMV_COL_U32)
    return fail(ISPMV_ERR_UNSUPPORTED, "plan from a device CSR: FP64/FP32 values, u32 columns");
  // the matrix is checked before any pass indexes through it
  DevTmp tmp;
  int *bad;
  UIN *flag, *pos;
  TRY(tmp.alloc(1, &bad));
  TRY(tmp.alloc((size_t)n + 1, &flag));
  TRY(tmp.alloc((size_t)n + 1, &pos));
  ISPMV_TRY(cudaMemsetAsync(bad, 0, sizeof(int), s));
  const unsigned gchk = (unsigned)std::min<size_t>(((size_t)std::max(n, nnz) + 255) / 256, (size_t)sm_count() * 16);
  dcsr_check<<<std::max(1u, gchk), 256, 0, s>>>(n, nnz, row, col, bad);
  TRY(check_launch("dcsr_check"));
  dcsr_flags<<<(unsigned)(((size_t)n + 1 + 255) / 256), 256, 0, s>>>(n, row, flag);
  TRY(check_launch("dcsr_flags"));
  size_t tb = 0;
  ISPMV_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag, pos, (int)n + 1, s));
  void *tst;
  TRY(tmp.alloc(tb, reinterpret_cast<unsigned char **>(&tst)));
  ISPMV_TRY(cub::DeviceScan::ExclusiveSum(tst, tb, flag, pos, (int)n + 1, s));
  int hbad = 0;
  UIN nonempty = 0;
  ISPMV_TRY(cudaMemcpyAsync(&hbad, bad, sizeof hbad, cudaMemcpyDeviceToHost, s));
  ISPMV_TRY(cudaMemcpyAsync(&nonempty, pos + n, sizeof nonempty, cudaMemcpyDeviceToHost, s));
  ISPMV_TRY(cudaStreamSynchronize(s));
  if (hbad) return fail(ISPMV_ERR_ARG, "plan from a device CSR: malformed row pointer or a column >= n");
  if (p->opts.kernel == ISPMV_KERNEL_AUTO) {
    // the compacted AXT's default (ispmv_plan_axt), with the scatter test
    // run on the device sample
    p->opts.kernel = ISPMV_KERNEL_WIDE;
    if (p->opts.variant == 0) {
      const bool long_rows = (double)nnz >= 16.0 * (double)n;
      bool scattered = false;
      const size_t S = std::min<size_t>(nnz, 1u << 16);
      if (S) {
        unsigned long long *dfar, hfar = 0;
        TRY(tmp.alloc(1, &dfar));
        ISPMV_TRY(cudaMemsetAsync(dfar, 0, sizeof *dfar, s));
        dcsr_far<<<(unsigned)((S + 255) / 256), 256, 0, s>>>(S, (double)nnz / (double)S, n, row, col, dfar);
        TRY(check_launch("dcsr_far"));
        ISPMV_TRY(cudaMemcpyAsync(&hfar, dfar, sizeof hfar, cudaMemcpyDeviceToHost, s));
        ISPMV_TRY(cudaStreamSynchronize(s));
        scattered = (double)hfar / (double)S >= 0.05;
      }
      p->opts.variant = auto_variant(p, long_rows, scattered);
    }
  }
  const WideCfg wc = wide_variant(p->opts.variant);
  if (!wc.ok || wc.tmem)
    return fail(ISPMV_ERR_UNSUPPORTED, "plan from a device CSR: the lane-interleaved kernel without TMEM staging");
  if (wc.stg && nnz > 0x7FFFFFFFu)
    return fail(ISPMV_ERR_UNSUPPORTED, "plan from a device CSR: per-CTA x windows up to 2^31 - 1 nonzeros");
  p->fmt = F_CSR;
  p->path = P_STREAM;
  p->n = n;
  p->nnz = nnz;
  p->slots = nnz;
  p->slots_pad = std::max(SS, (p->slots + SS - 1) / SS * SS);
  p->seg_slots = p->opts.units_per_warp <= 0 ? wc.seg : seg_slots_of(p, 1);
  if (p->seg_slots % SS) p->seg_slots = (p->seg_slots + SS - 1) / SS * SS;
  p->nseg = (p->slots_pad + p->seg_slots - 1) / p->seg_slots;
  const unsigned spl = (unsigned)wc.spl;
  void *vi;
  if (p->opts.val_kind == ISPMV_VAL_F64) TRY(dev_alloc(p, p->slots_pad, reinterpret_cast<double **>(&vi)));
  else TRY(dev_alloc(p, p->slots_pad, reinterpret_cast<float **>(&vi)));
  p->val = vi;
  TRY(dev_alloc(p, p->slots_pad, &p->col));
  TRY(dev_alloc(p, p->slots_pad / 32, &p->heads));
  TRY(dev_alloc(p, std::max<size_t>(1, p->nseg), &p->segh));
  p->nempty = n - nonempty;
  p->nrowmap = p->nempty ? nonempty : 0;
  if (p->nempty) {
    TRY(dev_alloc(p, p->nrowmap, &p->rowmap));
    TRY(dev_alloc(p, p->nempty, &p->empty));
  }
  ISPMV_TRY(cudaMemsetAsync(p->heads, 0, p->slots_pad / 32 * sizeof(UIN), s));
  const unsigned gi = (unsigned)std::min<size_t>((p->slots_pad + 255) / 256, (size_t)sm_count() * 32);
  if (p->opts.val_kind == ISPMV_VAL_F64)
    dcsr_interleave<double><<<gi, 256, 0, s>>>(nnz, p->slots_pad, spl, col, val, static_cast<double *>(vi), p->col);
  else
    dcsr_interleave<float><<<gi, 256, 0, s>>>(nnz, p->slots_pad, spl, col, val, static_cast<float *>(vi), p->col);
  TRY(check_launch("dcsr_interleave"));
  dcsr_rows<<<(unsigned)(((size_t)n + 255) / 256), 256, 0, s>>>(n, row, pos, p->heads, p->rowmap, p->empty);
  TRY(check_launch("dcsr_rows"));
  dcsr_segh<<<(unsigned)((p->nseg + 255) / 256), 256, 0, s>>>(p->nseg, p->seg_slots, n, row, pos, p->segh);
  TRY(check_launch("dcsr_segh"));
  size_t nt = 0;
  if (wc.stg) {
    // per-CTA x windows, as stage_windows picks them on the host
    const UIN W = wc.cap & ~1u, ne = n & ~1u;
    const size_t T = (size_t)WIDE_WARPS * p->seg_slots;
    nt = std::max<size_t>(1, (p->nseg + WIDE_WARPS - 1) / WIDE_WARPS);
    UIN *tlo, *tlen, *keys = nullptr, *sorted = nullptr;
    int *off;
    TRY(dev_alloc(p, nt, &tlo));
    TRY(dev_alloc(p, nt, &tlen));
    TRY(tmp.alloc(nt + 1, &off));
    dcsr_win_offsets<<<(unsigned)((nt + 1 + 255) / 256), 256, 0, s>>>(nt, T, nnz, off);
    TRY(check_launch("dcsr_win_offsets"));
    if (ne > W && nnz) {
      TRY(tmp.alloc(nnz, &keys));
      TRY(tmp.alloc(nnz, &sorted));
      dcsr_win_keys<<<gi, 256, 0, s>>>(nnz, col, val, keys);
      TRY(check_launch("dcsr_win_keys"));
      size_t sb = 0;
      ISPMV_TRY(cub::DeviceSegmentedRadixSort::SortKeys(nullptr, sb, keys, sorted, (int)nnz, (int)nt, off, off + 1,
                                                         0, 32, s));
      void *sst;
      TRY(tmp.alloc(sb, reinterpret_cast<unsigned char **>(&sst)));
      ISPMV_TRY(cub::DeviceSegmentedRadixSort::SortKeys(sst, sb, keys, sorted, (int)nnz, (int)nt, off, off + 1, 0, 32,
                                                         s));
    }
    dcsr_windows<<<(unsigned)nt, 256, 0, s>>>(nt, off, sorted, W, ne, tlo, tlen);
    TRY(check_launch("dcsr_windows"));
    p->xw.tlo = tlo;
    p->xw.tlen = tlen;
    p->xw.cap = W;
    p->xw.nwin = 1;
    p->xw.n = p->n;
  }
  TRY(alloc_records(p));
  if (wc.stg) p->xw.status = p->status;
  ISPMV_TRY(cudaStreamSynchronize(s));
  p->info.device_bytes = (uint64_t)(8 * nt) + (uint64_t)p->slots_pad * (vbytes(p) + 4) + p->slots_pad / 8;
  return ISPMV_OK;
}

}  // namespace

ISPMV_API int ispmv_plan_dev_csr(UIN n, UIN nnz, const UIN *d_row, const UIN *d_col, const FPT *d_val,
                                 const ispmv_plan_opts *o, ispmv_plan *out, void *stream) {
  if (!out || !d_row || n == 0 || (nnz && (!d_col || !d_val))) return ISPMV_ERR_ARG;
  if ((uint64_t)nnz + sss::SS > 0xFFFFFFFFull) return ISPMV_ERR_OVERFLOW;  // slot ids stay in 32 bits
  ispmv_plan_s *p;
  TRY(begin(o, &p));
  const int st = dev_csr_stream(p, n, nnz, d_row, d_col, d_val, as_stream(stream));
  finish_info(p, "CSR");
  return done(p, st, out);
}

ISPMV_API int ispmv_plan_get_layout(ispmv_plan p, ispmv_plan_layout *l) {
  if (!p || !l) return ISPMV_ERR_ARG;
  if (p->path != P_STREAM || p->opts.col_kind != ISPMV_COL_U32 ||
      (p->opts.kernel == ISPMV_KERNEL_WIDE && wide_variant(p->opts.variant).tmem))
    return ISPMV_ERR_UNSUPPORTED;
  std::memset(l, 0, sizeof *l);
  l->slots = p->slots;
  l->slots_pad = p->slots_pad;
  l->seg_slots = p->seg_slots;
  l->nseg = p->nseg;
  l->nrowmap = p->nrowmap;
  l->nempty = p->nempty;
  l->val_bytes = (UIN)vbytes(p);
  l->spl = p->opts.kernel == ISPMV_KERNEL_WIDE ? (UIN)wide_variant(p->opts.variant).spl : 0u;
  l->nwin = p->opts.kernel == ISPMV_KERNEL_WIDE && wide_variant(p->opts.variant).stg
                ? std::max<size_t>(1, (p->nseg + WIDE_WARPS - 1) / WIDE_WARPS)
                : 0;
  return ISPMV_OK;
}

ISPMV_API int ispmv_plan_export_windows(ispmv_plan p, UIN *lo, UIN *len, void *stream) {
  ispmv_plan_layout l;
  TRY(ispmv_plan_get_layout(p, &l));
  cudaStream_t s = as_stream(stream);
  if (l.nwin && lo) ISPMV_TRY(cudaMemcpyAsync(lo, p->xw.tlo, l.nwin * sizeof(UIN), cudaMemcpyDefault, s));
  if (l.nwin && len) ISPMV_TRY(cudaMemcpyAsync(len, p->xw.tlen, l.nwin * sizeof(UIN), cudaMemcpyDefault, s));
  ISPMV_TRY(cudaStreamSynchronize(s));
  return ISPMV_OK;
}

ISPMV_API int ispmv_plan_export_stream(ispmv_plan p, void *val, UIN *col, UIN *heads, UIN *segh, UIN *rowmap,
                                       UIN *empty, void *stream) {
  ispmv_plan_layout l;
  TRY(ispmv_plan_get_layout(p, &l));
  cudaStream_t s = as_stream(stream);
  auto cp = [&](void *dst, const void *src, size_t bytes) -> int {
    if (dst && src && bytes) ISPMV_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s));
    return ISPMV_OK;
  };
  TRY(cp(val, p->val, l.slots_pad * l.val_bytes));
  TRY(cp(col, p->col, l.slots_pad * sizeof(UIN)));
  TRY(cp(heads, p->heads, l.slots_pad / 32 * sizeof(UIN)));
  TRY(cp(segh, p->segh, l.nseg * sizeof(UIN)));
  TRY(cp(rowmap, p->rowmap, l.nrowmap * sizeof(UIN)));
  TRY(cp(empty, p->empty, l.nempty * sizeof(UIN)));
  ISPMV_TRY(cudaStreamSynchronize(s));
  return ISPMV_OK;
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
  std::vector<UIN> c(axi, axi + p->slots);
  for (size_t s = 0; s < p->slots; s++) v[s] = axc->ax[(s / 8) * 16 + s % 8];
  int st = ISPMV_OK;
  if (p->opts.kernel == ISPMV_KERNEL_AUTO) auto_wide(p, csr);  // the brick stream
  if (p->opts.kernel == ISPMV_KERNEL_ROWS) {
    // the reference's row loop (M:711-732): 8 lanes per row over its bricks
    if (narrow_kinds(p)) { ispmv_plan_destroy(p); return ISPMV_ERR_UNSUPPORTED; }
    p->opts.kernel = ISPMV_KERNEL_ROWS;
    p->path = P_ROWS;
    std::vector<UIN> bptr((size_t)p->n + 1);
    for (size_t r = 0; r <= p->n; r++) bptr[r] = axc->brp[r] / 16;
    st = upload_values(p, v);
    if (!st) st = dev_upload(p, c.data(), c.size(), &p->col);
    if (!st) st = dev_upload(p, bptr.data(), bptr.size(), &p->rows);
    p->info.device_bytes = (uint64_t)p->slots * (vbytes(p) + 4) + 4ull * (p->n + 1);
  } else {
    std::vector<size_t> start(p->n);
    for (UIN r = 0; r < p->n; r++) start[r] = axc->brp[r] / 2;
    st = setup_stream(p, csr, v, c, start);
  }
  finish_info(p, "AXC");
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
  if (narrow_kinds(p)) {
    delete p;
    return ISPMV_ERR_UNSUPPORTED;
  }
  p->fmt = reorder ? F_K1P : F_K1;
  p->path = P_K1;
  p->opts.kernel = ISPMV_KERNEL_ROWS;
  p->n = csr->nrows;
  p->nnz = csr->nnz;
  p->slots = k1->lenVC;
  p->chunkNum = k1->chunkNum;
  // the long chunks (a warp each): the prefix of chunks with at least
  // K1_LONG columns (nmc never increases: rows are sorted by length)
  p->k1_long = 0;
  while (p->k1_long < k1->chunkNum && k1->nmc[p->k1_long] >= K1_LONG) p->k1_long++;
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
  if (!axt || !axi || !axt->ax || !axt->sec || !axt->con || axt->nrows != csr->nrows) return ISPMV_ERR_ARG;
  if (axt->tileHW != 8 || axt->tileH == 0) return ISPMV_ERR_UNSUPPORTED;
  const bool com = std::strncmp(axt->mode, "COM", 3) == 0;
  const bool noc = std::strncmp(axt->mode, "NOC", 3) == 0;
  if (!com && !noc) return ISPMV_ERR_ARG;
  if (com && axt->tileH != 1) return ISPMV_ERR_UNSUPPORTED;
  ispmv_plan_s *p;
  TRY(begin(o, &p));
  if (p->opts.kernel == ISPMV_KERNEL_ROWS) {
    delete p;
    return ISPMV_ERR_UNSUPPORTED;
  }
  p->n = csr->nrows;
  p->nnz = csr->nnz;
  p->th = axt->tileH;
  p->fmt = com ? F_AXT_COM : F_AXT_NOC;
  char name[32];
  int st = ISPMV_OK;
  const UIN th = axt->tileH;
  if (com) {
    p->bs = 1u << axt->log;
    snprintf(name, sizeof name, "AXT_COM_BS%u", p->bs);
  } else {
    snprintf(name, sizeof name, "AXT_NOC_H%u", th);
  }
  // tileH > 1 on the slot-stream kernels: the tiles' slots in tile-column
  // order (tile, column, sub-row), where each row is one contiguous run
  const bool noc_stream = !com && th > 1 && (p->opts.kernel == ISPMV_KERNEL_AUTO || p->opts.kernel == ISPMV_KERNEL_WIDE);
  if (com || th == 1 || noc_stream) {
    // the tileH=1 tile stream and the packed compacted stream: every row is
    // a contiguous run of slots starting at the slot its con[] names; a
    // tileH > 1 tile (th sub-rows of 8 columns, a row filling columns top to
    // bottom, M:1188-1221) read column by column is such a stream too
    p->slots = com ? csr->nnz : (size_t)axt->lenAX / 2;
    std::vector<double> v(p->slots);
    std::vector<UIN> c(p->slots);
    std::vector<size_t> start(p->n);
    if (th == 1) {
      std::copy(axi, axi + p->slots, c.begin());
      for (size_t q = 0; q < p->slots; q++) v[q] = axt->ax[(q / 8) * 16 + q % 8];
      for (UIN r = 0; r < p->n; r++) start[r] = (size_t)(axt->con[r] / 16) * 8 + axt->con[r] % 16;
    } else {
      const size_t tile = (size_t)8 * th;  // value slots per tile
      for (size_t q = 0; q < p->slots; q++) {  // q: slot in ax order (tile, sub-row, column)
        const size_t T = q / tile, R = (q % tile) / 8, C = q % 8;
        const size_t sc = T * tile + C * th + R;  // the same slot in column order
        v[sc] = axt->ax[(q / 8) * 16 + q % 8];
        c[sc] = axi[q];
      }
      for (UIN r = 0; r < p->n; r++) {  // con = T*16*th + R*16 + C (M:1118-1148)
        const size_t T = axt->con[r] / (16 * th), rem = axt->con[r] % (16 * th);
        start[r] = T * tile + (rem % 16) * th + rem / 16;
      }
    }
    if (p->opts.kernel == ISPMV_KERNEL_AUTO) {
      // the lane-interleaved kernel: 8 slots per lane for rows of fewer than
      // 16 nonzeros on average, where the columns are scattered with per-CTA
      // x windows (FP64 values) or the next batch's columns loaded ahead
      // (FP32 values, whose kernel has the registers for it); else 16,
      // bulk-copy staged for FP64 values with u32 columns that are not
      // scattered (measured fastest there), plain loads for scattered columns
      // and for the FP32, lo-word and 16-bit-delta forms
      auto_wide(p, csr);
    }
    st = setup_stream(p, csr, v, c, start);
  } else {
    // tile columns: the unit engine on the reference's per-column rows
    p->path = P_UNITS;
    if (narrow_kinds(p)) st = ISPMV_ERR_UNSUPPORTED;
    size_t used = 0;
    for (UIN r = 0; r < p->n; r++) used += ((size_t)csr->rl[r] + th - 1) / th * th;
    p->slots = (size_t)axt->lenAX / 2;
    p->nunits = used / th;
    p->slots_pad = std::max(SS, (p->slots + SS - 1) / SS * SS);
    const bool regular = th == 4 || th == 8 || th == 16;
    if (p->opts.kernel == ISPMV_KERNEL_TMA && !regular) st = ISPMV_ERR_UNSUPPORTED;
    if (p->opts.kernel == ISPMV_KERNEL_AUTO) p->opts.kernel = ISPMV_KERNEL_LDG;
    if (regular) {
      p->seg_slots = seg_slots_of(p, th);
      p->useg = (UIN)(p->seg_slots / th);
      p->nseg = (p->slots_pad + p->seg_slots - 1) / p->seg_slots;
    } else {
      UIN u = p->opts.units_per_warp > 0 ? (UIN)p->opts.units_per_warp : std::max<UIN>(32u, (2048u / th) & ~31u);
      p->useg = std::max<UIN>(32u, u & ~31u);
      p->seg_slots = (size_t)p->useg * th;
      p->nseg = (p->nunits + p->useg - 1) / p->useg;
    }
    std::vector<double> v(p->slots_pad, 0.0);
    std::vector<UIN> c(p->slots_pad, 0);
    for (size_t q = 0; q < p->slots; q++) {
      v[q] = axt->ax[(q / 8) * 16 + q % 8];
      c[q] = axi[q];
    }
    if (!st) st = upload_values(p, v);
    if (!st) st = dev_upload(p, c.data(), c.size(), &p->col);
    std::vector<UIN> ur(std::max<size_t>(p->slots_pad / th, p->nunits) + 32, NO_ROW);
    std::copy(axt->sec, axt->sec + p->nunits, ur.begin());
    if (!st) st = dev_upload(p, ur.data(), ur.size(), &p->rows);
    if (!st) st = empty_rows(p, csr);
    if (!st) st = alloc_records(p);
    p->info.device_bytes = (uint64_t)p->slots_pad * (vbytes(p) + 4) + 4ull * p->nunits;
  }
  finish_info(p, name);
  return done(p, st, out);
}

ISPMV_API int ispmv_plan_get_info(ispmv_plan p, ispmv_plan_info *info) {
  if (!p || !info) return ISPMV_ERR_ARG;
  *info = p->info;
  return ISPMV_OK;
}

// ------------------------------------------------------------ execute --
namespace {

constexpr int TW = 4;  // warps per CTA of the staged kernels
constexpr int TS = 4;  // stages per warp

template <typename K>
int launch_staged(K kernel, size_t smem, size_t nseg, int ctas_per_sm, cudaStream_t s, const char *what,
                  void **args) {
  const size_t want = (nseg + TW - 1) / TW;
  const size_t cap = (size_t)sm_count() * (size_t)(ctas_per_sm > 0 ? ctas_per_sm : 2);
  const unsigned g = (unsigned)std::max<size_t>(1, std::min(want, cap));
  ISPMV_TRY(cudaFuncSetAttribute((const void *)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  ISPMV_TRY(cudaLaunchKernel((const void *)kernel, dim3(g), dim3(TW * 32), args, smem, s));
  return check_launch(what);
}

template <int W, typename K>
int launch_staged_w(K kernel, size_t smem, size_t nseg, int ctas_per_sm, cudaStream_t s, const char *what,
                    void **args) {
  const size_t want = (nseg + W - 1) / W;
  const size_t cap = (size_t)sm_count() * (size_t)ctas_per_sm;
  const unsigned g = (unsigned)std::max<size_t>(1, std::min(want, cap));
  ISPMV_TRY(cudaFuncSetAttribute((const void *)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  ISPMV_TRY(cudaLaunchKernel((const void *)kernel, dim3(g), dim3(W * 32), args, smem, s));
  return check_launch(what);
}

// A linear texture over `src` (bytes long, FP64 read as int2 or FP32),
// cached on the plan for the same buffer; 0 when the buffer does not meet
// the texture alignment or size limits (the caller then gathers with loads).
// Not inside graph capture: a later product with another x replaces the
// texture, which a captured graph would still name.
cudaTextureObject_t x_texture(ispmv_plan_s *p, const void *src, size_t bytes, bool f32) {
  if (p->capturing) return 0;
  if (p->xtex && p->xtex_src == src && p->xtex_bytes == bytes) return p->xtex;
  if (p->xtex) cudaDestroyTextureObject(p->xtex);
  p->xtex = 0;
  p->xtex_src = nullptr;
  int dev = 0, align = 0, maxw = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&align, cudaDevAttrTextureAlignment, dev) ||
      cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxTexture1DLinearWidth, dev))
    return 0;
  const size_t elems = bytes / (f32 ? 4 : 8);
  if (align <= 0 || reinterpret_cast<uintptr_t>(src) % (uintptr_t)align || elems > (size_t)maxw || elems >= (1u << 31))
    return 0;
  cudaResourceDesc rd{};
  rd.resType = cudaResourceTypeLinear;
  rd.res.linear.devPtr = const_cast<void *>(src);
  rd.res.linear.desc = f32 ? cudaCreateChannelDesc<float>() : cudaCreateChannelDesc<int2>();
  rd.res.linear.sizeInBytes = bytes;
  cudaTextureDesc td{};
  td.readMode = cudaReadModeElementType;
  if (cudaCreateTextureObject(&p->xtex, &rd, &td, nullptr) != cudaSuccess) {
    cudaGetLastError();
    p->xtex = 0;
    return 0;
  }
  p->xtex_src = src;
  p->xtex_bytes = bytes;
  return p->xtex;
}

template <typename VT, int SPL, int MINB, bool D16 = false, bool TEX = false, bool STG = false, bool LO = false,
          bool PFC = false>
int launch_wide(ispmv_plan_s *p, const FPT *x, seg::Out &o, cudaStream_t s, const char *name) {
  constexpr int NW = STG ? 1 : 0;
  if constexpr (sizeof(VT) == 4 && !STG && !LO) {
    // FP32 values: gather from an FP32 copy of x (the value the FP32 multiply uses)
    if (!p->x32) TRY(dev_alloc(p, p->n, &p->x32));
    const unsigned gc = (unsigned)std::min<size_t>(((size_t)p->n / 2 + 255) / 256, (size_t)sm_count() * 8) + 1;
    if ((reinterpret_cast<uintptr_t>(x) & 15u) == 0) wide::x_to_f32<true><<<gc, 256, 0, s>>>(p->n, x, p->x32);
    else wide::x_to_f32<false><<<gc, 256, 0, s>>>(p->n, x, p->x32);
    TRY(check_launch("x_to_f32"));
    const cudaTextureObject_t tx = TEX ? x_texture(p, p->x32, (size_t)p->n * 4, true) : 0;
    if (TEX && !tx) return launch_wide<VT, SPL, MINB, D16, false>(p, x, o, s, "stream_wide<tex: x gathered with loads>");
    // a programmatic dependent of x_to_f32: its CTAs load their first
    // batch while x is rounded, and wait for x_to_f32 before they gather
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((p->nseg + WIDE_WARPS - 1) / WIDE_WARPS));
    cfg.blockDim = dim3(WIDE_WARPS * 32);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    ISPMV_TRY(cudaLaunchKernelEx(&cfg, wide::stream_wide<VT, float, SPL, 0, WIDE_WARPS, MINB, D16, TEX, false, false, PFC>,
                                 p->slots, p->slots_pad, p->seg_slots, p->nseg, static_cast<const VT *>(p->val),
                                 (const UIN *)p->col, (const UIN *)p->heads, (const UIN *)p->segh, p->xw,
                                 (const float *)p->x32, o, p->narrow, tx));
    return check_launch(name);
  } else {
    const cudaTextureObject_t tx = TEX ? x_texture(p, x, (size_t)p->n * 8, false) : 0;
    if (TEX && !tx) return launch_wide<VT, SPL, MINB, D16, false>(p, x, o, s, "stream_wide<tex: x gathered with loads>");
    auto *k = wide::stream_wide<VT, double, SPL, NW, WIDE_WARPS, MINB, D16, TEX, STG, LO, PFC>;
    const size_t smem = STG ? (size_t)p->xw.cap * sizeof(double) : 0;
    if (smem) ISPMV_TRY(cudaFuncSetAttribute((const void *)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const unsigned g = (unsigned)((p->nseg + WIDE_WARPS - 1) / WIDE_WARPS);
    k<<<g, WIDE_WARPS * 32, smem, s>>>(p->slots, p->slots_pad, p->seg_slots, p->nseg, static_cast<const VT *>(p->val),
                                        p->col, p->heads, p->segh, p->xw, x, o, p->narrow, tx);
    return check_launch(name);
  }
}

// The staged form: persistent, as many CTAs as fit on the SMs (at most one
// warp per segment).
template <typename VT, int SPL, int STAGES, int W>
int launch_wide_tma(ispmv_plan_s *p, const FPT *x, seg::Out &o, cudaStream_t s, const char *name) {
  auto *k = wide::stream_wide_tma<VT, SPL, STAGES, W>;
  const size_t smem = wide::tma_smem_bytes<VT, SPL, STAGES, W>();
  ISPMV_TRY(cudaFuncSetAttribute((const void *)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  ISPMV_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, W * 32, smem));
  if (p->opts.ctas_per_sm > 0) per_sm = std::min(per_sm, p->opts.ctas_per_sm);
  const size_t want = (p->nseg + W - 1) / W;
  const unsigned g = (unsigned)std::max<size_t>(1, std::min(want, (size_t)sm_count() * (size_t)std::max(1, per_sm)));
  k<<<g, W * 32, smem, s>>>(p->slots, p->slots_pad, p->seg_slots, p->nseg, static_cast<const VT *>(p->val), p->col,
                            p->heads, p->segh, x, o, p->status);
  return check_launch(name);
}

// The TMEM-staged form: one CTA of 4 consumer warps + 1 producer warp per 4
// segments.
template <typename VT, int SPL, int S, int H>
int launch_tmem(ispmv_plan_s *p, const FPT *x, seg::Out &o, cudaStream_t s, const char *name) {
  const void *xs = x;
  if constexpr (sizeof(VT) == 4) {  // FP32 values: gather the FP32 copy of x
    if (!p->x32) TRY(dev_alloc(p, p->n, &p->x32));
    const unsigned gc = (unsigned)std::min<size_t>(((size_t)p->n / 2 + 255) / 256, (size_t)sm_count() * 8) + 1;
    if ((reinterpret_cast<uintptr_t>(x) & 15u) == 0) wide::x_to_f32<true><<<gc, 256, 0, s>>>(p->n, x, p->x32);
    else wide::x_to_f32<false><<<gc, 256, 0, s>>>(p->n, x, p->x32);
    TRY(check_launch("x_to_f32"));
    xs = p->x32;
  }
  using XT = typename std::conditional<sizeof(VT) == 4, float, double>::type;
  auto *k = tmemk::stream_tmem<VT, XT, SPL, S, H>;
  const size_t smem = tmemk::smem_bytes<VT, SPL, S, H>();
  ISPMV_TRY(cudaFuncSetAttribute((const void *)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const unsigned g = (unsigned)(p->nseg / (tmemk::CW * H));
  k<<<g, (tmemk::CW * H + 1) * 32, smem, s>>>(p->slots, p->seg_slots, p->tblocks, p->heads, p->segh,
                                               static_cast<const XT *>(xs), o, p->status);
  return check_launch(name);
}

template <typename VT>
int run_wide(ispmv_plan_s *p, const FPT *x, seg::Out &o, cudaStream_t s) {
  const WideCfg wc = wide_variant(p->opts.variant);
  if (wc.tmem) {
    switch (p->opts.variant) {
      case 18: return launch_tmem<VT, 8, 4, 1>(p, x, o, s, "stream_tmem<8,s4,w4>");
      case 19: return launch_tmem<VT, 16, 2, 1>(p, x, o, s, "stream_tmem<16,s2,w4>");
      case 20: return launch_tmem<VT, 8, 2, 2>(p, x, o, s, "stream_tmem<8,s2,w8>");
      default: return launch_tmem<VT, 16, 2, 2>(p, x, o, s, "stream_tmem<16,s2,w8>");
    }
  }
  if (wc.tma) return launch_wide_tma<VT, 16, 2, 4>(p, x, o, s, "stream_wide_tma<16,s2,w4>");
  const bool d = p->opts.col_kind == ISPMV_COL_D16;
  if constexpr (sizeof(VT) == 4) {
    if (p->opts.val_kind == ISPMV_VAL_F32_LO16) {  // plain loads, FP64 x (setup checks)
      if (wc.spl == 8)
        return d ? launch_wide<VT, 8, 4, true, false, false, true>(p, x, o, s, "stream_wide<8,w0,b4,d16,lo>")
                 : launch_wide<VT, 8, 4, false, false, false, true>(p, x, o, s, "stream_wide<8,w0,b4,lo>");
      return d ? launch_wide<VT, 16, 3, true, false, false, true>(p, x, o, s, "stream_wide<16,w0,b3,d16,lo>")
               : launch_wide<VT, 16, 3, false, false, false, true>(p, x, o, s, "stream_wide<16,w0,b3,lo>");
    }
  }
  if (wc.pfc)  // u32 columns (setup checks)
    return launch_wide<VT, 8, 4, false, false, false, false, true>(p, x, o, s, "stream_wide<8,w0,b4,pfc>");
  if (wc.stg) {
    if ((reinterpret_cast<uintptr_t>(x) & 15u) == 0)
      return launch_wide<VT, 8, 4, false, false, true>(p, x, o, s, "stream_wide<8,stg,b4>");
    // x not 16-byte aligned (no bulk copy): plain loads over the same stream
    return launch_wide<VT, 8, 4>(p, x, o, s, "stream_wide<8,w0,b4>");
  }
  if (wc.tex)  // texture gathers (loads where x does not fit a texture)
    return d ? launch_wide<VT, 8, 4, true, true>(p, x, o, s, "stream_wide<8,w0,b4,d16,tex>")
             : launch_wide<VT, 8, 4, false, true>(p, x, o, s, "stream_wide<8,w0,b4,tex>");
  if (wc.spl == 8)
    return d ? launch_wide<VT, 8, 4, true>(p, x, o, s, "stream_wide<8,w0,b4,d16>")
             : launch_wide<VT, 8, 4>(p, x, o, s, "stream_wide<8,w0,b4>");
  return d ? launch_wide<VT, 16, 3, true>(p, x, o, s, "stream_wide<16,w0,b3,d16>")
           : launch_wide<VT, 16, 3>(p, x, o, s, "stream_wide<16,w0,b3>");
}

template <typename VT>
int run_stream(ispmv_plan_s *p, const FPT *x, seg::Out &o, cudaStream_t s) {
  if (p->opts.kernel == ISPMV_KERNEL_WIDE) return run_wide<VT>(p, x, o, s);
  const VT *val = static_cast<const VT *>(p->val);
  size_t nslots = p->slots, spad = p->slots_pad, sslots = p->seg_slots, nseg = p->nseg;
  const UIN *col = p->col, *heads = p->heads, *segh = p->segh;
  if (narrow_kinds(p)) {
    const unsigned g = (unsigned)((nseg * 32 + 255) / 256);
    const bool lo = p->opts.val_kind == ISPMV_VAL_F32_LO16, d16 = p->opts.col_kind == ISPMV_COL_D16;
    if (lo && d16)
      sss::stream_narrow<VT, true, true><<<g, 256, 0, s>>>(nslots, spad, sslots, nseg, val, col, heads, segh, p->narrow, x, o);
    else if (lo)
      sss::stream_narrow<VT, true, false><<<g, 256, 0, s>>>(nslots, spad, sslots, nseg, val, col, heads, segh, p->narrow, x, o);
    else
      sss::stream_narrow<VT, false, true><<<g, 256, 0, s>>>(nslots, spad, sslots, nseg, val, col, heads, segh, p->narrow, x, o);
    return check_launch("stream_narrow");
  }
  if (p->opts.kernel == ISPMV_KERNEL_TMA) {
    int *status = p->status;
    void *args[] = {&nslots, &spad, &sslots, &nseg, &val, &col, &heads, &segh, (void *)&x, &o, &status};
    const int cps = p->opts.ctas_per_sm;
    // 8 warps per CTA, 2 stages of 256 slots per warp; CTAs per SM from shared memory
    return launch_staged_w<8>(sss::stream_tma<VT, 8, 2, 256>, sss::smem_bytes<8, 2, VT, 256>(), nseg,
                              cps ? cps : 4, s, "stream_tma<8,2,256>", args);
  }
  if (p->opts.variant == ISPMV_VARIANT_QUEUE) {
    ISPMV_TRY(cudaMemsetAsync(p->queue, 0, sizeof(unsigned long long), s));
    const size_t warps = std::min<size_t>(nseg, (size_t)sm_count() * 6 * 8);
    const unsigned gq = (unsigned)std::max<size_t>(1, (warps + 7) / 8);
    sss::stream_queue<VT><<<gq, 256, 0, s>>>(nslots, spad, sslots, nseg, val, col, heads, segh, x, p->queue, o);
    return check_launch("stream_queue");
  }
  const unsigned g = (unsigned)((nseg * 32 + 255) / 256);
  // variants: slots per lane x prefetch depth (batches in flight) x CTAs per
  // SM the register budget allows; the default (variant 0) is (4, 0, 5)
  const char *nm = "stream_ldg";
#define ISPMV_SSS(SPL, PD, MINB)                                                                              \
  sss::stream_ldg<VT, SPL, PD, MINB><<<g, 256, 0, s>>>(nslots, spad, sslots, nseg, val, col, heads, segh, x, o); \
  nm = "stream_ldg<" #SPL "," #PD "," #MINB ">";                                                                \
  break
#define ISPMV_SSS_PF(SPL, PD, MINB, PF)                                                              \
  sss::stream_ldg<VT, SPL, PD, MINB, PF><<<g, 256, 0, s>>>(nslots, spad, sslots, nseg, val, col, heads, segh, x, \
                                                           o);                                                   \
  nm = "stream_ldg<" #SPL "," #PD "," #MINB ",pf" #PF ">";                                                      \
  break
  switch (p->opts.variant) {
    case 2: ISPMV_SSS(4, 0, 6);
    case 12: ISPMV_SSS_PF(4, 0, 6, 2);
    default: ISPMV_SSS(4, 0, 5);
  }
#undef ISPMV_SSS
#undef ISPMV_SSS_PF
  return check_launch(nm);
}

template <typename VT>
int run_units(ispmv_plan_s *p, const FPT *x, seg::Out &o, cudaStream_t s) {
  const VT *val = static_cast<const VT *>(p->val);
  if (p->opts.kernel == ISPMV_KERNEL_TMA) {
    using L = tk::StageLayout<VT>;
    size_t nunits = p->nunits, spad = p->slots_pad, nseg = p->nseg, sslots = p->seg_slots;
    const UIN *col = p->col, *urow = p->rows;
    int *status = p->status;
    void *args[] = {&nunits, &spad, &nseg, &sslots, &val, &col, &urow, (void *)&x, &o, &status};
    const int cps = p->opts.ctas_per_sm;
    switch (p->th) {
      case 4:
        return launch_staged(tk::nocn_tma<VT, 4, TW, TS>, tk::smem_bytes<TW, TS>(L::VB + L::CB + (tk::SS / 4) * 4),
                             nseg, cps, s, "nocn_tma<4>", args);
      case 8:
        return launch_staged(tk::nocn_tma<VT, 8, TW, TS>, tk::smem_bytes<TW, TS>(L::VB + L::CB + (tk::SS / 8) * 4),
                             nseg, cps, s, "nocn_tma<8>", args);
      case 16:
        return launch_staged(tk::nocn_tma<VT, 16, TW, TS>,
                             tk::smem_bytes<TW, TS>(L::VB + L::CB + (tk::SS / 16) * 4), nseg, cps, s, "nocn_tma<16>",
                             args);
      default:
        return ISPMV_ERR_UNSUPPORTED;
    }
  }
  const unsigned g = (unsigned)((p->nseg * 32 + pk::TPB - 1) / pk::TPB);
  pk::noc_hn<VT><<<g, pk::TPB, 0, s>>>(p->nunits, p->nseg, p->th, p->useg, p->rows, p->col, val, x, o);
  return check_launch("noc_hn");
}

// Kernel timing marks: `which` 0 before the main kernel of a product, 1 after it.
int tmark(ispmv_plan_s *p, cudaStream_t s, int which) {
  if (!p->tcap || p->capturing) return ISPMV_OK;
  const size_t i = p->tcount % p->tcap;
  ISPMV_TRY(cudaEventRecord(p->tev[2 * i + which], s));
  if (which) p->tcount++;
  return ISPMV_OK;
}

template <typename VT>
int run_main(ispmv_plan_s *p, const FPT *x, FPT *y, int beta, cudaStream_t s);

template <typename VT>
int run(ispmv_plan_s *p, const FPT *x, FPT *y, int beta, cudaStream_t s) {
  TRY(tmark(p, s, 0));
  const int st = run_main<VT>(p, x, y, beta, s);
  if (st) return st;
  p->kname = last_launch();
  // the kernels after the main one (the row fix-up, K1's reorder)
  // the kernel after the main one is a programmatic dependent launch when
  // nothing (a timing event) sits between the two in the stream
  const bool pdl = !p->tcap || p->capturing;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  if (p->path == P_STREAM || p->path == P_UNITS) {
    TRY(tmark(p, s, 1));
    const size_t nrec = p->slots ? 2 * p->nseg : 0;
    const size_t work = std::max(nrec, p->nempty);
    if (work) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)((work + 255) / 256));
      cfg.blockDim = dim3(256);
      cfg.dynamicSmemBytes = 0;
      cfg.stream = s;
      cfg.attrs = at;
      cfg.numAttrs = pdl ? 1 : 0;
      ISPMV_TRY(cudaLaunchKernelEx(&cfg, seg::fixup, nrec, (const UIN *)p->rec_row, (const double *)p->rec_sum,
                                   (const UIN *)p->rowmap, (const UIN *)p->empty, p->nempty, y, beta));
      return check_launch("fixup");
    }
    return ISPMV_OK;
  }
  if (p->path == P_K1 && p->fmt != F_K1P) {
    TRY(tmark(p, s, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((p->n + 255) / 256));
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    ISPMV_TRY(cudaLaunchKernelEx(&cfg, pk::k1_order, p->n, (const UIN *)p->permi, (const FPT *)p->res, y, beta));
    return check_launch("k1_order");
  }
  return tmark(p, s, 1);
}

// The main kernel of one product.
template <typename VT>
int run_main(ispmv_plan_s *p, const FPT *x, FPT *y, int beta, cudaStream_t s) {
  const VT *val = static_cast<const VT *>(p->val);
  switch (p->path) {
    case P_ROWS: {
      if (p->fmt == F_AXC) {
        const unsigned g = (unsigned)(((size_t)p->n * 8 + pk::TPB - 1) / pk::TPB);
        pk::axc_rows<VT><<<g, pk::TPB, 0, s>>>(p->n, p->rows, p->col, val, x, y, beta);
        return check_launch("axc_rows");
      }
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
    case P_K1: {
      const unsigned g = (unsigned)((pk::k1_warps(p->chunkNum, p->k1_long) * 32 + pk::TPB - 1) / pk::TPB);
      if (p->fmt == F_K1P) {
        pk::k1_chunks<VT, true><<<g, pk::TPB, 0, s>>>(p->n, p->chunkNum, p->k1_long, p->chp, p->nmc, p->permi,
                                                      p->col, val, x, y, beta);
        return check_launch("k1_chunks<scatter>");
      }
      pk::k1_chunks<VT, false><<<g, pk::TPB, 0, s>>>(p->n, p->chunkNum, p->k1_long, p->chp, p->nmc, p->permi,
                                                     p->col, val, x, p->res, beta);
      return check_launch("k1_chunks");
    }
    case P_STREAM:
    case P_UNITS: {
      seg::Out o{y, p->rowmap, p->rec_row, p->rec_sum, beta};
      if (p->slots) TRY(p->path == P_STREAM ? run_stream<VT>(p, x, o, s) : run_units<VT>(p, x, o, s));
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

ISPMV_API int ispmv_plan_spmv_graph(ispmv_plan p, const FPT *x, FPT *y, int beta, void *stream) {
  if (!p || !x || !y || (beta != 0 && beta != 1)) return ISPMV_ERR_ARG;
  if (!p->graph_exec || p->g_x != x || p->g_y != y || p->g_beta != beta) {
    if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    p->graph_exec = nullptr;
    p->graph = nullptr;
    if (!p->cap_stream) ISPMV_TRY(cudaStreamCreateWithFlags(&p->cap_stream, cudaStreamNonBlocking));
    // work areas a product allocates on first use, allocated before the
    // capture (no allocation may happen inside it): the FP32 copy of x of
    // FP32-value plans on the lane-interleaved kernel
    if (p->opts.val_kind != ISPMV_VAL_F64 && p->opts.kernel == ISPMV_KERNEL_WIDE && !p->x32)
      TRY(dev_alloc(p, p->n, &p->x32));
    ISPMV_TRY(cudaStreamBeginCapture(p->cap_stream, cudaStreamCaptureModeThreadLocal));
    p->capturing = true;
    const int st = p->opts.val_kind == ISPMV_VAL_F64 ? run<double>(p, x, y, beta, p->cap_stream)
                                                     : run<float>(p, x, y, beta, p->cap_stream);
    p->capturing = false;
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(p->cap_stream, &g);
    if (st || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      // a failed capture leaves its error as the runtime's last error: clear
      // it so that it is not reported again by a later, unrelated call
      (void)cudaGetLastError();
      return st ? st : cuda_status(e, "cudaStreamEndCapture");
    }
    p->graph = g;
    ISPMV_TRY(cudaGraphInstantiate(&p->graph_exec, p->graph, 0));
    p->g_x = x;
    p->g_y = y;
    p->g_beta = beta;
  }
  ISPMV_TRY(cudaGraphLaunch(p->graph_exec, as_stream(stream)));
  count_launch();
  return ISPMV_OK;
}

ISPMV_API int ispmv_plan_time_kernels(ispmv_plan p, int pairs) {
  if (!p || pairs < 0) return ISPMV_ERR_ARG;
  for (cudaEvent_t e : p->tev) cudaEventDestroy(e);
  p->tev.clear();
  p->tcap = 0;
  p->tcount = 0;
  for (int i = 0; i < 2 * pairs; i++) {
    cudaEvent_t e;
    ISPMV_TRY(cudaEventCreate(&e));
    p->tev.push_back(e);
  }
  p->tcap = (size_t)pairs;
  return ISPMV_OK;
}

ISPMV_API int ispmv_plan_kernel_ms(ispmv_plan p, double *total_ms, int *launches) {
  if (!p || !total_ms || !launches) return ISPMV_ERR_ARG;
  const size_t m = std::min(p->tcount, p->tcap);
  double sum = 0.0;
  for (size_t i = 0; i < m; i++) {
    float ms = 0.f;
    ISPMV_TRY(cudaEventElapsedTime(&ms, p->tev[2 * i], p->tev[2 * i + 1]));
    sum += ms;
  }
  *total_ms = sum;
  *launches = (int)m;
  p->tcount = 0;
  return ISPMV_OK;
}

ISPMV_API int ispmv_plan_time_main(ispmv_plan p, const FPT *x, FPT *y, int reps, void *stream, double *ms) {
  if (!p || !x || !y || reps < 1 || !ms) return ISPMV_ERR_ARG;
  if (p->capturing) return fail(ISPMV_ERR_ARG, "ispmv_plan_time_main: not inside a graph capture");
  cudaStream_t s = as_stream(stream);
  auto ck = [](cudaError_t e, const char *where) { return e == cudaSuccess ? ISPMV_OK : cuda_status(e, where); };
  cudaEvent_t e[2] = {nullptr, nullptr};
  ISPMV_TRY(cudaEventCreate(&e[0]));
  int st = ck(cudaEventCreate(&e[1]), "cudaEventCreate");
  if (!st) st = ck(cudaEventRecord(e[0], s), "cudaEventRecord");
  for (int i = 0; i < reps && !st; i++)
    st = p->opts.val_kind == ISPMV_VAL_F64 ? run_main<double>(p, x, y, 0, s) : run_main<float>(p, x, y, 0, s);
  if (!st) st = ck(cudaEventRecord(e[1], s), "cudaEventRecord");
  if (!st) st = ck(cudaEventSynchronize(e[1]), "cudaEventSynchronize");
  float t = 0.f;
  if (!st) st = ck(cudaEventElapsedTime(&t, e[0], e[1]), "cudaEventElapsedTime");
  for (cudaEvent_t ev : e)
    if (ev) cudaEventDestroy(ev);
  if (!st) *ms = (double)t / reps;
  return st;
}

ISPMV_API const char *ispmv_plan_kernel_name(ispmv_plan p) { return p ? p->kname : ""; }

ISPMV_API int ispmv_plan_status(ispmv_plan p) {
  if (!p) return ISPMV_ERR_ARG;
  if (!p->status) return ISPMV_OK;
  int v = 0;
  ISPMV_TRY(cudaMemcpy(&v, p->status, sizeof v, cudaMemcpyDeviceToHost));
  return v;
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
  return ispmv_plan_status(p);
}

namespace {
// Slots per lane of a lane-interleaved (stream_wide) plan, 0 for slot order.
unsigned il_spl(const ispmv_plan_s *p) {
  return p->opts.kernel == ISPMV_KERNEL_WIDE ? (unsigned)wide_variant(p->opts.variant).spl : 0u;
}
bool tmem_plan(const ispmv_plan_s *p) {
  return p->opts.kernel == ISPMV_KERNEL_WIDE && wide_variant(p->opts.variant).tmem;
}

// One pass per block of CB = G*W right-hand sides (G lanes per group, W
// columns per lane).
template <int G, int W, typename VT, int SPL>
int spmm_blocks(ispmv_plan_s *p, UIN k, const FPT *X, FPT *Y, cudaStream_t s) {
  constexpr int NG = 32 / G, CB = G * W;
  const size_t nparts = p->nseg * NG, nrec = 2 * nparts;
  if (p->mm_rows_cap < nrec) {
    TRY(dev_alloc(p, std::max<size_t>(1, nrec), &p->mm_row));
    p->mm_rows_cap = nrec;
  }
  if (p->mm_cap < nrec * CB) {
    TRY(dev_alloc(p, std::max<size_t>(1, nrec * CB), &p->mm_sum));
    p->mm_cap = nrec * CB;
  }
  const VT *val = static_cast<const VT *>(p->val);
  for (UIN j0 = 0; j0 < k; j0 += CB) {
    mm::Out o{Y, p->rowmap, p->mm_row, p->mm_sum, k, j0, std::min<UIN>(CB, k - j0)};
    const unsigned g = (unsigned)((p->nseg * 32 + 255) / 256);
    mm::stream_spmm<G, W, VT, SPL><<<g, 256, 0, s>>>(p->slots, p->slots_pad, p->seg_slots, p->nseg, val, p->col,
                                                     p->heads, p->segh, X, o);
    TRY(check_launch("stream_spmm"));
    p->kname = last_launch();
    const size_t work = std::max(nrec, p->nempty) * CB;
    mm::spmm_fixup<CB><<<(unsigned)((work + 255) / 256), 256, 0, s>>>(nrec, p->mm_row, p->mm_sum, p->empty,
                                                                      p->nempty, o);
    TRY(check_launch("spmm_fixup"));
  }
  return ISPMV_OK;
}

// Four columns per lane: one pass per block of CB = 4G right-hand sides.
template <int G, int T, int MINB, typename VT, int SPL>
int spmm_blocks4(ispmv_plan_s *p, UIN k, const FPT *X, FPT *Y, cudaStream_t s) {
  constexpr int NG = 32 / G, CB = 4 * G;
  const size_t nparts = p->nseg * NG, nrec = 2 * nparts;
  if (p->mm_rows_cap < nrec) {
    TRY(dev_alloc(p, std::max<size_t>(1, nrec), &p->mm_row));
    p->mm_rows_cap = nrec;
  }
  if (p->mm_cap < nrec * CB) {
    TRY(dev_alloc(p, std::max<size_t>(1, nrec * CB), &p->mm_sum));
    p->mm_cap = nrec * CB;
  }
  const VT *val = static_cast<const VT *>(p->val);
  for (UIN j0 = 0; j0 < k; j0 += CB) {
    mm::Out o{Y, p->rowmap, p->mm_row, p->mm_sum, k, j0, std::min<UIN>(CB, k - j0)};
    const unsigned g = (unsigned)((p->nseg * 32 + 255) / 256);
    mm::stream_spmm4<G, T, MINB, VT, SPL><<<g, 256, 0, s>>>(p->slots, p->slots_pad, p->seg_slots, p->nseg, val,
                                                            p->col, p->heads, p->segh, X, o);
    TRY(check_launch("stream_spmm4"));
    p->kname = last_launch();
    const size_t work = std::max(nrec, p->nempty) * CB;
    mm::spmm_fixup<CB><<<(unsigned)((work + 255) / 256), 256, 0, s>>>(nrec, p->mm_row, p->mm_sum, p->empty,
                                                                      p->nempty, o);
    TRY(check_launch("spmm_fixup"));
  }
  return ISPMV_OK;
}

// RHS block 8, 16 or 32 columns (ispmv_plan_opts.rhs_block, else by k).
// spmm_kernel: WIDE four columns per lane with 32-byte X loads (k a
// multiple of 4, X and Y 32-byte aligned); LDG two columns per lane (4, 8 or 16
// lanes per group); AUTO the four-column form for blocks of 16 and 32
// columns where it applies, else two (on 8-column blocks the two-column
// form is the faster with FP64 values).
template <typename VT, int SPL>
int spmm_run_spl(ispmv_plan_s *p, UIN k, const FPT *X, FPT *Y, cudaStream_t s) {
  int g = p->opts.rhs_block;
  if (g != 8 && g != 16 && g != 32) g = k <= 8 ? 8 : k <= 16 ? 16 : 32;
  const bool four_ok = (k & 3u) == 0 && ((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(Y)) & 31u) == 0;
  const int kind = p->opts.spmm_kernel;
  if (kind == ISPMV_KERNEL_WIDE && !four_ok)
    return fail(ISPMV_ERR_UNSUPPORTED,
                "ispmv_plan_spmm: four columns per lane need k a multiple of 4 and X, Y 32-byte aligned");
  if (four_ok && (kind == ISPMV_KERNEL_WIDE || (kind == ISPMV_KERNEL_AUTO && g > 8))) {
    if (g == 8) return spmm_blocks4<2, 8, 2, VT, SPL>(p, k, X, Y, s);
    if (g == 16) return spmm_blocks4<4, 4, 3, VT, SPL>(p, k, X, Y, s);
    return spmm_blocks4<8, 8, 2, VT, SPL>(p, k, X, Y, s);
  }
  if (g == 8) return spmm_blocks<4, 2, VT, SPL>(p, k, X, Y, s);
  if (g == 16) return spmm_blocks<8, 2, VT, SPL>(p, k, X, Y, s);
  return spmm_blocks<16, 2, VT, SPL>(p, k, X, Y, s);
}

// The plan's stream layout as a template argument: slot order, or lane-
// interleaved with 8 or 16 slots per lane.
template <typename VT>
int spmm_run(ispmv_plan_s *p, UIN k, const FPT *X, FPT *Y, cudaStream_t s) {
  switch (il_spl(p)) {
    case 0: return spmm_run_spl<VT, 0>(p, k, X, Y, s);
    case 8: return spmm_run_spl<VT, 8>(p, k, X, Y, s);
    case 16: return spmm_run_spl<VT, 16>(p, k, X, Y, s);
    default: return fail(ISPMV_ERR_UNSUPPORTED, "ispmv_plan_spmm: lane-interleaved plans of 8 or 16 slots per lane");
  }
}
}  // namespace

// Y = A X for k right-hand sides (row-major n x k): the slot-stream plans
// (AXT COM, AXT tileH=1, AXC and CSR built with the stream kernels).
ISPMV_API int ispmv_plan_spmm(ispmv_plan p, UIN k, const FPT *X, FPT *Y, void *stream) {
  if (!p || !X || !Y || k == 0) return ISPMV_ERR_ARG;
  if (p->path != P_STREAM || narrow_kinds(p) || tmem_plan(p))
    return fail(ISPMV_ERR_UNSUPPORTED, "ispmv_plan_spmm: needs a slot-stream plan with u32 columns");
  cudaStream_t s = as_stream(stream);
  if (!p->slots) {  // every row empty
    ISPMV_TRY(cudaMemsetAsync(Y, 0, (size_t)p->n * k * sizeof(FPT), s));
    return ISPMV_OK;
  }
  if (p->opts.val_kind == ISPMV_VAL_F64) return spmm_run<double>(p, k, X, Y, s);
  return spmm_run<float>(p, k, X, Y, s);
}
