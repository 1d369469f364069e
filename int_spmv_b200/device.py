"""Device side: the reference's kernels by name on CUDA tensors, and plans.

`int_axc`, `int_k1`, ... run the sm_100a kernels of libintspmv.so on the
reference's own arrays (x-baked ax included), stream-ordered on the current
torch stream, with each reference kernel's output contract (AXT kernels
accumulate into y: zero it first, as the reference's callers do,
intSpmv_main.c:1421,1492,1591).

`Plan` uploads a format once and computes y = A x (+ beta y) for a fresh x on
every call (values FP64, or FP32 with FP64 accumulation).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import abi
from ._lib import check, load
from .formats import AXC, AXT, CSR, K1


def _ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t.data_ptr()


def _stream(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def to_device(a: np.ndarray, device="cuda") -> torch.Tensor:
    """u32 arrays travel as int32 tensors (same bits); f64 as float64."""
    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32)).to(device)
    return torch.from_numpy(np.ascontiguousarray(a)).to(device)


# --- the reference's kernels on device tensors (intSpmv_main.c line cited) ---

def cf_CSR(row, col, val, x, y, stream=None):  # :382
    check(load().ispmv_dev_cf_csr(row.numel() - 1, _ptr(row), _ptr(col), _ptr(val), _ptr(x), _ptr(y),
                                  _stream(stream)), "ispmv_dev_cf_csr")


def int_axc(nrows, ax, brp, y, stream=None):  # :711
    check(load().ispmv_dev_int_axc(nrows, _ptr(ax), _ptr(brp), _ptr(y), _stream(stream)), "ispmv_dev_int_axc")


def int_k1(chunkNum, val, col, chp, nmc, vec, res, stream=None):  # :943
    check(load().ispmv_dev_int_k1(chunkNum, _ptr(val), _ptr(col), _ptr(chp), _ptr(nmc), _ptr(vec), _ptr(res),
                                  _stream(stream)), "ispmv_dev_int_k1")


def orderArrayK1(length, permi, arrDis, arrOrd, stream=None):  # :969
    check(load().ispmv_dev_order_k1(length, _ptr(permi), _ptr(arrDis), _ptr(arrOrd), _stream(stream)),
          "ispmv_dev_order_k1")


def int_k1p(mask, chunkNum, val, col, chp, nmc, permi, vec, res, stream=None):  # :1026
    check(load().ispmv_dev_int_k1p(mask, chunkNum, _ptr(val), _ptr(col), _ptr(chp), _ptr(nmc), _ptr(permi),
                                   _ptr(vec), _ptr(res), _stream(stream)), "ispmv_dev_int_k1p")


def int_axt_noc_h1(tileNum, ax, rwp, y, stream=None):  # :1385
    check(load().ispmv_dev_int_axt_noc_h1(tileNum, _ptr(ax), _ptr(rwp), _ptr(y), _stream(stream)),
          "ispmv_dev_int_axt_noc_h1")


def int_axt_noc(tileNum, tileHeight, ax, rwp, y, stream=None):  # :1443
    check(load().ispmv_dev_int_axt_noc(tileNum, tileHeight, _ptr(ax), _ptr(rwp), _ptr(y), _stream(stream)),
          "ispmv_dev_int_axt_noc")


def int_axt_com_h1(bn, bs, log, thw, tn, lenAX, lenRWP, ax, rwp, y, stream=None):  # :1517
    check(load().ispmv_dev_int_axt_com_h1(bn, bs, log, thw, tn, lenAX, lenRWP, _ptr(ax), _ptr(rwp), _ptr(y),
                                          _stream(stream)), "ispmv_dev_int_axt_com_h1")


# --- plans ---

VAL_KINDS = {"f64": abi.VAL_F64, "f32": abi.VAL_F32, "f32lo": abi.VAL_F32_LO16}
COL_KINDS = {"u32": abi.COL_U32, "d16": abi.COL_D16}
KERNELS = {"auto": abi.KERNEL_AUTO, "ldg": abi.KERNEL_LDG, "tma": abi.KERNEL_TMA, "rows": abi.KERNEL_ROWS,
           "wide": abi.KERNEL_WIDE}


def plan_opts(val="f64", col="u32", kernel="auto", units_per_warp=0, ctas_per_sm=0, lo_tol=0.0,
              variant=0, rhs_block=0, spmm_kernel="auto") -> abi.PlanOpts:
    o = abi.PlanOpts()
    load().ispmv_plan_opts_default(C.byref(o))
    o.val_kind, o.col_kind, o.kernel = VAL_KINDS[val], COL_KINDS[col], KERNELS[kernel]
    o.units_per_warp, o.ctas_per_sm, o.lo_tol, o.variant = units_per_warp, ctas_per_sm, lo_tol, variant
    o.rhs_block, o.spmm_kernel = rhs_block, KERNELS[spmm_kernel]
    return o


class Plan:
    """A format resident in HBM.  `fmt` is the host format object built by
    int_spmv_b200.formats (None for CSR); K1 takes `reorder` (True = int_k1p,
    False = int_k1 then orderArrayK1)."""

    def __init__(self, csr: CSR, fmt: AXC | K1 | AXT | None = None, *, reorder: bool = True, val="f64", col="u32",
                 kernel="auto", units_per_warp=0, ctas_per_sm=0, lo_tol=0.0, variant=0, rhs_block=0,
                 spmm_kernel="auto", axi: np.ndarray | None = None):
        lib = load()
        o = plan_opts(val, col, kernel, units_per_warp, ctas_per_sm, lo_tol, variant, rhs_block, spmm_kernel)
        h = C.c_void_p()
        if fmt is None:
            check(lib.ispmv_plan_csr(C.byref(csr.c), C.byref(o), C.byref(h)), "ispmv_plan_csr")
        elif isinstance(fmt, AXC):
            axi = fmt.cols() if axi is None else axi
            check(lib.ispmv_plan_axc(C.byref(csr.c), C.byref(fmt.c), axi.ctypes.data_as(abi.P_UIN), C.byref(o),
                                     C.byref(h)), "ispmv_plan_axc")
        elif isinstance(fmt, K1):
            check(lib.ispmv_plan_k1(C.byref(csr.c), C.byref(fmt.c), int(reorder), C.byref(o), C.byref(h)),
                  "ispmv_plan_k1")
        elif isinstance(fmt, AXT):
            axi = fmt.cols() if axi is None else axi
            check(lib.ispmv_plan_axt(C.byref(csr.c), C.byref(fmt.c), axi.ctypes.data_as(abi.P_UIN), C.byref(o),
                                     C.byref(h)), "ispmv_plan_axt")
        else:
            raise TypeError(f"unsupported format {type(fmt)}")
        self._h = h
        self.n = csr.n
        self.nnz = csr.nnz

    @classmethod
    def from_device_csr(cls, row: torch.Tensor, col: torch.Tensor, val: torch.Tensor, *, val_kind="f64",
                        kernel="auto", variant=0, units_per_warp=0, stream=None) -> "Plan":
        """The compacted AXT's slot stream built on the GPU from CSR arrays
        already in device memory (ispmv_plan_dev_csr; u32 arrays as int32
        tensors): the same arrays as Plan(csr, kernel="wide", variant=...)
        builds on the host.  Raises IntSpmvError on a malformed CSR."""
        n, nnz = row.numel() - 1, col.numel()
        if n < 1 or val.numel() != nnz or val.dtype != torch.float64:
            raise ValueError("expected row (n+1), col (nnz) and float64 val (nnz) CUDA tensors")
        o = plan_opts(val_kind, "u32", kernel, units_per_warp, 0, 0.0, variant, 0)
        h = C.c_void_p()
        check(load().ispmv_plan_dev_csr(n, nnz, _ptr(row), _ptr(col) if nnz else None, _ptr(val) if nnz else None,
                                        C.byref(o), C.byref(h), _stream(stream)), "ispmv_plan_dev_csr")
        self = cls.__new__(cls)
        self._h, self.n, self.nnz = h, n, nnz
        return self

    def export_stream(self, stream=None) -> dict:
        """The slot-stream plan's device arrays as numpy arrays (values as
        raw bytes), with the layout's lengths."""
        lib = load()
        lay = abi.PlanLayout()
        check(lib.ispmv_plan_get_layout(self._h, C.byref(lay)), "ispmv_plan_get_layout")
        a = dict(val=np.zeros(lay.slots_pad * lay.val_bytes, np.uint8), col=np.zeros(lay.slots_pad, np.uint32),
                 heads=np.zeros(lay.slots_pad // 32, np.uint32), segh=np.zeros(lay.nseg, np.uint32),
                 rowmap=np.zeros(lay.nrowmap, np.uint32), empty=np.zeros(lay.nempty, np.uint32))
        p = {k: (v.ctypes.data if v.size else None) for k, v in a.items()}
        check(lib.ispmv_plan_export_stream(self._h, p["val"], p["col"], p["heads"], p["segh"], p["rowmap"],
                                           p["empty"], _stream(stream)), "ispmv_plan_export_stream")
        a["win_lo"], a["win_len"] = np.zeros(lay.nwin, np.uint32), np.zeros(lay.nwin, np.uint32)
        if lay.nwin:
            check(lib.ispmv_plan_export_windows(self._h, a["win_lo"].ctypes.data, a["win_len"].ctypes.data,
                                                _stream(stream)), "ispmv_plan_export_windows")
        a["layout"] = {f: getattr(lay, f) for f, _ in abi.PlanLayout._fields_}
        return a

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                load().ispmv_plan_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def info(self) -> dict:
        i = abi.PlanInfo()
        check(load().ispmv_plan_get_info(self._h, C.byref(i)), "ispmv_plan_get_info")
        return dict(nrows=i.nrows, nnz=i.nnz, slots=i.slots, device_bytes=i.device_bytes, alg_bytes=i.alg_bytes,
                    format=i.format, val_kind=i.val_kind, col_kind=i.col_kind, kernel=i.kernel, tile_h=i.tile_h,
                    bs=i.bs, name=i.name.decode())

    def status(self) -> int:
        """ISPMV_ERR_TIMEOUT if a bounded device wait gave up, else 0 (syncs)."""
        return int(load().ispmv_plan_status(self._h))

    def time_kernels(self, pairs: int) -> None:
        """Record a CUDA event pair around the main kernel of each spmv
        (a ring of `pairs`; 0 turns it off)."""
        check(load().ispmv_plan_time_kernels(self._h, int(pairs)), "ispmv_plan_time_kernels")

    def kernel_ms(self) -> tuple[float, int]:
        """(summed main-kernel milliseconds, pairs) since the last call; the
        stream must be synchronised first."""
        ms, n = C.c_double(), C.c_int()
        check(load().ispmv_plan_kernel_ms(self._h, C.byref(ms), C.byref(n)), "ispmv_plan_kernel_ms")
        return ms.value, n.value

    def time_main(self, x: torch.Tensor, y: torch.Tensor, reps: int, stream=None) -> float:
        """Mean milliseconds of the main kernel over `reps` back-to-back
        launches between one CUDA event pair (ispmv_plan_time_main); y is
        left without the row fix-up (run spmv for the product)."""
        if x.dtype != torch.float64 or x.numel() != self.n or y.numel() != self.n:
            raise ValueError("x and y must be float64 CUDA tensors of n entries")
        ms = C.c_double()
        check(load().ispmv_plan_time_main(self._h, _ptr(x), _ptr(y), int(reps), _stream(stream), C.byref(ms)),
              "ispmv_plan_time_main")
        return ms.value

    def kernel_name(self) -> str:
        """The main kernel of the latest product (e.g. "stream_ldg<4,0,5>")."""
        return load().ispmv_plan_kernel_name(self._h).decode()

    def spmv(self, x: torch.Tensor, y: torch.Tensor | None = None, beta: int = 0, stream=None) -> torch.Tensor:
        if x.dtype != torch.float64 or x.numel() != self.n:
            raise ValueError("x must be a float64 CUDA tensor of n entries")
        if y is None:
            y = torch.empty(self.n, dtype=torch.float64, device=x.device)
        check(load().ispmv_plan_spmv(self._h, _ptr(x), _ptr(y), int(beta), _stream(stream)), "ispmv_plan_spmv")
        return y

    def spmv_graph(self, x: torch.Tensor, y: torch.Tensor, beta: int = 0, stream=None) -> torch.Tensor:
        """spmv as one CUDA-graph launch (captured on first use for these x, y)."""
        check(load().ispmv_plan_spmv_graph(self._h, _ptr(x), _ptr(y), int(beta), _stream(stream)),
              "ispmv_plan_spmv_graph")
        return y

    def spmm(self, X: torch.Tensor, Y: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        if X.dtype != torch.float64 or X.dim() != 2 or X.shape[0] != self.n:
            raise ValueError("X must be a float64 CUDA tensor of shape (n, k)")
        k = X.shape[1]
        if Y is None:
            Y = torch.empty((self.n, k), dtype=torch.float64, device=X.device)
        check(load().ispmv_plan_spmm(self._h, k, _ptr(X), _ptr(Y), _stream(stream)), "ispmv_plan_spmm")
        return Y

    def spmv_host(self, x: np.ndarray | torch.Tensor, y: np.ndarray | torch.Tensor, stream=None) -> None:
        """End to end on host buffers (pinned host tensors for full PCIe
        bandwidth): copy x in, SpMV, copy y out, synchronise."""
        xp = x.data_ptr() if isinstance(x, torch.Tensor) else x.ctypes.data
        yp = y.data_ptr() if isinstance(y, torch.Tensor) else y.ctypes.data
        check(load().ispmv_plan_spmv_host(self._h, xp, yp, _stream(stream)), "ispmv_plan_spmv_host")


# --- format conversion on the GPU ---

class DeviceAXT:
    """getFormatDataAXT (intSpmv_main.c:1275) run on the GPU
    (ispmv_dev_build_axt): con, the x-baked ax and sec of the AXT format, bit
    for bit the host builder's, built from CSR arrays and x already on the
    device (u32 arrays as int32 tensors).  The arrays stay in device memory
    (owned here); `fd` is the format data with the GPU conversion time."""

    def __init__(self, row: torch.Tensor, col: torch.Tensor, val: torch.Tensor, x: torch.Tensor, bs: int = 128,
                 thw: int = 8, th: int = 1, mode: str = "COM", stream=None):
        lib = load()
        n, nnz = row.numel() - 1, col.numel()
        self.c, self.fd = abi.StrMatAXT(), abi.StrFormatData()
        check(lib.ispmv_dev_build_axt(bs, thw, th, mode.encode(), n, nnz, _ptr(row), _ptr(col) if nnz else None,
                                      _ptr(val) if nnz else None, _ptr(x), C.byref(self.c), C.byref(self.fd),
                                      _stream(stream)), "ispmv_dev_build_axt")

    def __del__(self):
        c = getattr(self, "c", None)
        if c is not None and c.ax:
            try:
                load().ispmv_dev_axt_free(C.byref(c))
            except Exception:
                pass

    @property
    def conversion_s(self) -> float:
        return float(self.fd.ct)

    def to_host(self, stream=None) -> dict:
        """con, ax and sec copied to numpy arrays."""
        con = np.zeros(self.c.lenCON, np.uint32)
        ax = np.zeros(self.c.lenAX, np.float64)
        sec = np.zeros(self.c.lenSEC, np.uint32)
        check(load().ispmv_dev_axt_export(C.byref(self.c), con.ctypes.data or None, ax.ctypes.data or None,
                                          sec.ctypes.data or None, _stream(stream)), "ispmv_dev_axt_export")
        return dict(con=con, ax=ax, sec=sec)

    def spmv(self, y: torch.Tensor, stream=None) -> torch.Tensor:
        """The reference kernel of this AXT (int_axt_noc_h1, int_axt_noc or
        int_axt_com_h1) on the device arrays; like the reference it
        accumulates into y (zero it first)."""
        lib, c = load(), self.c
        ax, sec = C.cast(c.ax, C.c_void_p), C.cast(c.sec, C.c_void_p)
        mode = c.mode.decode()
        if mode == "NOC" and c.tileH == 1:
            check(lib.ispmv_dev_int_axt_noc_h1(c.tileN, ax, sec, _ptr(y), _stream(stream)), "ispmv_dev_int_axt_noc_h1")
        elif mode == "NOC":
            check(lib.ispmv_dev_int_axt_noc(c.tileN, c.tileH, ax, sec, _ptr(y), _stream(stream)),
                  "ispmv_dev_int_axt_noc")
        else:
            bs = 1 << c.log
            bn = (c.lenSEC + bs - 1) // bs  # blocks of bs slots (intSpmv_main.c:1517)
            check(lib.ispmv_dev_int_axt_com_h1(bn, bs, c.log, c.tileHW, c.tileN, c.lenAX, c.lenSEC, ax, sec, _ptr(y),
                                               _stream(stream)), "ispmv_dev_int_axt_com_h1")
        return y


class DeviceK1:
    """getFormatDataK1 (intSpmv_main.c:841) run on the GPU
    (ispmv_dev_build_k1): permi, nmc, chp, val and col of the K1 format, bit
    for bit the host builder's, from CSR arrays on the device; the arrays stay
    in device memory (owned here)."""

    def __init__(self, row: torch.Tensor, col: torch.Tensor, val: torch.Tensor, stream=None):
        lib = load()
        n, nnz = row.numel() - 1, col.numel()
        self.c, self.fd = abi.StrMatK1(), abi.StrFormatData()
        check(lib.ispmv_dev_build_k1(n, nnz, _ptr(row), _ptr(col) if nnz else None, _ptr(val) if nnz else None,
                                     C.byref(self.c), C.byref(self.fd), _stream(stream)), "ispmv_dev_build_k1")

    def __del__(self):
        c = getattr(self, "c", None)
        if c is not None and c.permi:
            try:
                load().ispmv_dev_k1_free(C.byref(c))
            except Exception:
                pass

    @property
    def conversion_s(self) -> float:
        return float(self.fd.ct)

    def to_host(self, stream=None) -> dict:
        cn, lv = self.c.chunkNum, self.c.lenVC
        a = dict(permi=np.zeros((cn + 1) * 8, np.uint32), nmc=np.zeros(cn, np.uint32), chp=np.zeros(cn, np.uint32),
                 val=np.zeros(lv, np.float64), col=np.zeros(lv, np.uint32))
        ptr = {k: (v.ctypes.data or None) for k, v in a.items()}
        check(load().ispmv_dev_k1_export(C.byref(self.c), ptr["permi"], ptr["nmc"], ptr["chp"], ptr["val"],
                                         ptr["col"], _stream(stream)), "ispmv_dev_k1_export")
        return a

    def spmv(self, x: torch.Tensor, y: torch.Tensor, stream=None) -> torch.Tensor:
        """int_k1p (K1 with integrated reordering, intSpmv_main.c:1026) on
        the device arrays: y[permi[i]] = row i of the chunk order."""
        c = self.c
        rem = c.nrows - 8 * (c.chunkNum - 1)
        mask = (1 << rem) - 1
        vp = lambda q: C.cast(q, C.c_void_p)  # noqa: E731
        check(load().ispmv_dev_int_k1p(mask, c.chunkNum, vp(c.val), vp(c.col), vp(c.chp), vp(c.nmc), vp(c.permi),
                                       _ptr(x), _ptr(y), _stream(stream)), "ispmv_dev_int_k1p")
        return y
