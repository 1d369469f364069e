"""Host formats with the reference's interface (edoardoCB/int_spmv,
intSpmv_main.c): `getFormatDataCSR/AXC/K1/AXT` build a format from a CSR
matrix and return the reference's (str_formatData, struct) pair, `getErrors`
and `initVec` as in the reference.  Arrays are allocated by the C builders
(libintspmv.so) and freed when the Python object is collected; numpy views of
them stay valid only while their owner lives.  Errors raise IntSpmvError
where the reference exits (intSpmv_main.c:171-179)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import abi
from ._lib import check, load

U32, F64 = np.uint32, np.float64


def _view(ptr, n: int, dtype):
    if n == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).view(dtype)


def _p(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


@dataclass
class FormatData:
    """str_formatData (intSpmv_main.c:306): name, memory footprint [B],
    occupancy beta, conversion time [s]."""
    name: str
    mfp: float
    beta: float
    ct: float

    @classmethod
    def of(cls, fd: abi.StrFormatData) -> "FormatData":
        return cls(fd.name.decode(), fd.mfp, fd.beta, fd.ct)


class CSR:
    """str_matCSR (intSpmv_main.c:183) over numpy arrays; `rl` and the row
    statistics are filled at construction (the stats pass, M:253-278)."""

    def __init__(self, row, col, val, nrows: int | None = None):
        self.row = np.ascontiguousarray(row, dtype=U32)
        self.col = np.ascontiguousarray(col, dtype=U32)
        self.val = np.ascontiguousarray(val, dtype=F64)
        n = len(self.row) - 1 if nrows is None else nrows
        self.rl = np.zeros(max(n, 1), dtype=U32)
        s = abi.StrMatCSR()
        s.nrows, s.nnz = n, len(self.col)
        s.val, s.row, s.col, s.rl = _p(self.val, C.c_double), _p(self.row, C.c_uint), _p(self.col, C.c_uint), \
            _p(self.rl, C.c_uint)
        self.c = s
        check(load().ispmv_csr_stats(C.byref(s)), "ispmv_csr_stats")

    @property
    def n(self) -> int:
        return self.c.nrows

    @property
    def nnz(self) -> int:
        return self.c.nnz

    def stats(self) -> dict:
        s = self.c
        return dict(nrows=s.nrows, nnz=s.nnz, rmin=s.rmin, rave=s.rave, rmax=s.rmax, rsd=s.rsd, bw=s.bw)

    @classmethod
    def read(cls, path: str) -> "CSR":
        """matrixReading (intSpmv_main.c:187-249): .csr text or .bin file."""
        s = abi.StrMatCSR()
        lib = load()
        check(lib.ispmv_matrix_read(str(path).encode(), C.byref(s)), f"ispmv_matrix_read({path})")
        try:
            n, nnz = s.nrows, s.nnz
            row = _view(s.row, n + 1, U32).copy()
            col = _view(s.col, nnz, U32).copy()
            val = _view(s.val, nnz, F64).copy()
        finally:
            lib.ispmv_csr_free(C.byref(s))
        return cls(row, col, val)

    def write(self, path: str) -> None:
        check(load().ispmv_matrix_write(str(path).encode(), C.byref(self.c)), f"ispmv_matrix_write({path})")


class _Owned:
    _free = ""

    def __del__(self):
        try:
            if getattr(self, "c", None) is not None:
                getattr(load(), self._free)(C.byref(self.c))
        except Exception:
            pass


class AXC(_Owned):
    """str_matAXC (intSpmv_main.c:615)."""
    _free = "ispmv_free_axc"

    def __init__(self, c: abi.StrMatAXC, csr: CSR):
        self.c, self._csr = c, csr
        self.ax = _view(c.ax, c.lenAX, F64)
        self.brp = _view(c.brp, c.lenBRP, U32)

    def cols(self, ompNT: int = 0) -> np.ndarray:
        """Column companion of ax's value slots (no reference counterpart)."""
        p = C.POINTER(C.c_uint)()
        check(load().ispmv_build_axc_cols(ompNT, C.byref(self._csr.c), C.byref(self.c), C.byref(p)),
              "ispmv_build_axc_cols")
        return _take_malloced(p, self.c.lenAX // 2)


class K1(_Owned):
    """str_matK1 (intSpmv_main.c:771)."""
    _free = "ispmv_free_k1"

    def __init__(self, c: abi.StrMatK1, csr: CSR):
        self.c, self._csr = c, csr
        self.permi = _view(c.permi, (c.chunkNum + 1) * 8, U32)
        self.nmc = _view(c.nmc, c.chunkNum, U32)
        self.chp = _view(c.chp, c.chunkNum, U32)
        self.val = _view(c.val, c.lenVC, F64)
        self.col = _view(c.col, c.lenVC, U32)

    @property
    def mask(self) -> int:
        """Tail mask of the last chunk (intSpmv_main.c:1077-1086)."""
        return 0xFF >> (self.c.chunkNum * 8 - self.c.nrows)


class AXT(_Owned):
    """str_matAXT (intSpmv_main.c:1114)."""
    _free = "ispmv_free_axt"

    def __init__(self, c: abi.StrMatAXT, csr: CSR):
        self.c, self._csr = c, csr
        self.ax = _view(c.ax, c.lenAX, F64)
        self.sec = _view(c.sec, c.lenSEC, U32)
        self.con = _view(c.con, c.lenCON, U32)

    @property
    def mode(self) -> str:
        return self.c.mode.decode()

    def cols(self, ompNT: int = 0) -> np.ndarray:
        p = C.POINTER(C.c_uint)()
        check(load().ispmv_build_axt_cols(ompNT, C.byref(self._csr.c), C.byref(self.c), C.byref(p)),
              "ispmv_build_axt_cols")
        return _take_malloced(p, self.c.lenAX // 2)


def _take_malloced(p, n: int) -> np.ndarray:
    out = _view(p, n, U32).copy()
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    libc.free(C.cast(p, C.c_void_p))
    return out


def _vec_ptr(vec: np.ndarray):
    vec = np.ascontiguousarray(vec, dtype=F64)
    return vec, _p(vec, C.c_double)


def getFormatDataCSR(csr: CSR) -> FormatData:
    """getFormatDataCSR (intSpmv_main.c:324-357)."""
    fd = abi.StrFormatData()
    check(load().ispmv_build_csr(C.byref(csr.c), C.byref(fd)), "getFormatDataCSR")
    return FormatData.of(fd)


def getFormatDataAXC(ompNT: int, csr: CSR, vec) -> tuple[FormatData, AXC]:
    """getFormatDataAXC (intSpmv_main.c:662-707)."""
    vec, vp = _vec_ptr(vec)
    m, fd = abi.StrMatAXC(), abi.StrFormatData()
    check(load().ispmv_build_axc(ompNT, C.byref(csr.c), vp, C.byref(m), C.byref(fd)), "getFormatDataAXC")
    return FormatData.of(fd), AXC(m, csr)


def getFormatDataK1(blockSize: int, csr: CSR, vec) -> tuple[FormatData, K1]:
    """getFormatDataK1 (intSpmv_main.c:841-905)."""
    vec, vp = _vec_ptr(vec)
    m, fd = abi.StrMatK1(), abi.StrFormatData()
    check(load().ispmv_build_k1(blockSize, C.byref(csr.c), vp, C.byref(m), C.byref(fd)), "getFormatDataK1")
    return FormatData.of(fd), K1(m, csr)


def getFormatDataAXT(ompNT: int, bs: int, thw: int, th: int, mode: str, csr: CSR, vec) -> tuple[FormatData, AXT]:
    """getFormatDataAXT (intSpmv_main.c:1275-1381)."""
    vec, vp = _vec_ptr(vec)
    m, fd = abi.StrMatAXT(), abi.StrFormatData()
    check(load().ispmv_build_axt(ompNT, bs, thw, th, mode.encode(), C.byref(csr.c), vp, C.byref(m), C.byref(fd)),
          f"getFormatDataAXT({mode}, th={th}, bs={bs})")
    return FormatData.of(fd), AXT(m, csr)


def getErrors(ref: np.ndarray, res: np.ndarray) -> tuple[float, float, int]:
    """getErrors (intSpmv_main.c:404-425): (aErr, rErr, pos)."""
    ref = np.ascontiguousarray(ref, dtype=F64)
    res = np.ascontiguousarray(res, dtype=F64)
    e = abi.StrErr()
    load().getErrors(len(ref), _p(ref, C.c_double), _p(res, C.c_double), C.byref(e))
    return e.aErr, e.rErr, e.pos


def initVec(n: int) -> np.ndarray:
    """initVec (intSpmv_main.c:361-367): x[i] = i."""
    v = np.empty(n, dtype=F64)
    load().initVec(n, _p(v, C.c_double))
    return v
