"""TEST INFRASTRUCTURE ONLY - Python access to the two checkers:

  Oracle     oracle.c, the C restatement of the reference's algorithms
             (oracle/_build/liboracle.so);
  Reference  the reference itself (edoardoCB/int_spmv intSpmv_main.c compiled
             from its own source by oracle/Makefile into
             oracle/_ref/libintspmv_ref.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs use this module, and only as checkers.  The product package
(int_spmv_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from int_spmv_b200 import abi

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libintspmv_ref.so"
U32, F64 = np.uint32, np.float64
P_U, P_D = C.POINTER(C.c_uint), C.POINTER(C.c_double)


# Where this build environment keeps the reference checkout when
# $INTSPMV_REF_DIR does not name one (read only by this build step).
_REF_CHECKOUT = "/root/reference"


def ref_dir() -> str | None:
    """The reference checkout to compile oracle/_ref from: $INTSPMV_REF_DIR,
    else the build environment's checkout when present, else None (a
    prebuilt oracle/_ref is then kept, as on a machine without the source)."""
    d = os.environ.get("INTSPMV_REF_DIR") or _REF_CHECKOUT
    return d if os.path.exists(os.path.join(d, "intSpmv_main.c")) else None


def build(quiet: bool = True) -> None:
    """make -C oracle: the restatement always, the reference when its source
    is present (otherwise a prebuilt _ref library is kept)."""
    cmd = ["make", "-C", str(HERE)]
    rd = ref_dir()
    if rd:
        cmd.append(f"REF_DIR={rd}")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    if not quiet:
        print(r.stdout)


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _u(a):
    return np.ascontiguousarray(a, dtype=U32)


def _d(a):
    return np.ascontiguousarray(a, dtype=F64)


class Oracle:
    """The C restatement (oracle.c)."""

    def __init__(self):
        if not ORACLE_SO.exists():
            build()
        self.lib = C.CDLL(str(ORACLE_SO))

    # M:253-278
    def stats(self, row, col):
        row, col = _u(row), _u(col)
        n = len(row) - 1
        rl = np.zeros(n, U32)
        rmin, rmax, bw = C.c_uint(), C.c_uint(), C.c_uint()
        rave, rsd = C.c_double(), C.c_double()
        self.lib.orc_stats(C.c_uint(n), _p(row, C.c_uint), _p(col, C.c_uint), _p(rl, C.c_uint), C.byref(rmin),
                           C.byref(rave), C.byref(rmax), C.byref(rsd), C.byref(bw))
        return dict(rl=rl, rmin=rmin.value, rave=rave.value, rmax=rmax.value, rsd=rsd.value, bw=bw.value)

    # M:382-396
    def cf_csr(self, row, col, val, x):
        row, col, val, x = _u(row), _u(col), _d(val), _d(x)
        n = len(row) - 1
        y = np.zeros(n, F64)
        self.lib.orc_cf_csr(C.c_uint(n), _p(row, C.c_uint), _p(col, C.c_uint), _p(val, C.c_double),
                            _p(x, C.c_double), _p(y, C.c_double))
        return y

    def abs_csr(self, row, col, val, x):
        row, col, val, x = _u(row), _u(col), _d(val), _d(x)
        n = len(row) - 1
        y = np.zeros(n, F64)
        self.lib.orc_abs_csr(C.c_uint(n), _p(row, C.c_uint), _p(col, C.c_uint), _p(val, C.c_double),
                             _p(x, C.c_double), _p(y, C.c_double))
        return y

    # M:404-425
    def get_errors(self, ref, res):
        ref, res = _d(ref), _d(res)
        a, r, pos = C.c_double(), C.c_double(), C.c_uint()
        self.lib.orc_get_errors(C.c_uint(len(ref)), _p(ref, C.c_double), _p(res, C.c_double), C.byref(a),
                                C.byref(r), C.byref(pos))
        return a.value, r.value, pos.value

    # AXC, M:619-658
    def axc(self, row, col, val, x, rl):
        row, col, val, x, rl = _u(row), _u(col), _d(val), _d(x), _u(rl)
        n = len(rl)
        brp = np.zeros(n + 1, U32)
        self.lib.orc_axc_brp.restype = C.c_uint
        lenax = self.lib.orc_axc_brp(C.c_uint(n), _p(rl, C.c_uint), _p(brp, C.c_uint))
        ax = np.zeros(lenax, F64)
        self.lib.orc_axc_ax(C.c_uint(n), _p(row, C.c_uint), _p(col, C.c_uint), _p(val, C.c_double),
                            _p(x, C.c_double), _p(brp, C.c_uint), _p(ax, C.c_double))
        return dict(brp=brp, ax=ax, lenAX=lenax)

    def axc_spmv(self, ax, brp):
        ax, brp = _d(ax), _u(brp)
        n = len(brp) - 1
        y = np.zeros(n, F64)
        self.lib.orc_axc_spmv(C.c_uint(n), _p(ax, C.c_double), _p(brp, C.c_uint), _p(y, C.c_double))
        return y

    # K1, M:775-837
    def k1(self, row, col, val, rl):
        row, col, val, rl = _u(row), _u(col), _d(val), _u(rl)
        n = len(rl)
        cn = (n + 7) // 8
        permi = np.zeros((cn + 1) * 8, U32)
        if self.lib.orc_k1_permi(C.c_uint(n), _p(rl, C.c_uint), _p(permi, C.c_uint)) != 0:
            raise MemoryError("orc_k1_permi")
        nmc, chp = np.zeros(cn, U32), np.zeros(cn, U32)
        self.lib.orc_k1_nmc_chp.restype = C.c_uint
        lenvc = self.lib.orc_k1_nmc_chp(C.c_uint(n), _p(rl, C.c_uint), _p(permi, C.c_uint), _p(nmc, C.c_uint),
                                        _p(chp, C.c_uint))
        kval, kcol = np.zeros(lenvc, F64), np.zeros(lenvc, U32)
        self.lib.orc_k1_valcol(C.c_uint(n), _p(row, C.c_uint), _p(col, C.c_uint), _p(val, C.c_double),
                               _p(permi, C.c_uint), _p(chp, C.c_uint), _p(kval, C.c_double), _p(kcol, C.c_uint))
        return dict(permi=permi, nmc=nmc, chp=chp, val=kval, col=kcol, chunkNum=cn, lenVC=lenvc)

    def k1_spmv(self, k, x):
        x = _d(x)
        cn = k["chunkNum"]
        res = np.zeros(cn * 8, F64)
        self.lib.orc_k1_spmv(C.c_uint(cn), _p(k["val"], C.c_double), _p(k["col"], C.c_uint), _p(k["chp"], C.c_uint),
                             _p(k["nmc"], C.c_uint), _p(x, C.c_double), _p(res, C.c_double))
        return res

    def k1_order(self, permi, res, n):
        ord_ = np.zeros(n, F64)
        res = _d(res)
        permi = _u(permi)
        self.lib.orc_k1_order(C.c_uint(n), _p(permi, C.c_uint), _p(res, C.c_double), _p(ord_, C.c_double))
        return ord_

    def k1p_spmv(self, k, x, n):
        x = _d(x)
        y = np.zeros(n + 1, F64)
        self.lib.orc_k1p_spmv(C.c_uint(n), C.c_uint(k["chunkNum"]), _p(k["val"], C.c_double), _p(k["col"], C.c_uint),
                              _p(k["chp"], C.c_uint), _p(k["nmc"], C.c_uint), _p(k["permi"], C.c_uint),
                              _p(x, C.c_double), _p(y, C.c_double))
        return y[:n]

    # AXT, M:1118-1260
    def axt(self, row, col, val, x, rl, thw, th, mode, bs=128):
        row, col, val, x, rl = _u(row), _u(col), _d(val), _d(x), _u(rl)
        n = len(rl)
        noc = mode == "NOC"
        con = np.zeros(n, U32)
        out = np.zeros(3, U32)
        self.lib.orc_axt_len(C.c_uint(n), _p(rl, C.c_uint), C.c_uint(thw), C.c_uint(th), C.c_int(int(noc)),
                             _p(con, C.c_uint), _p(out, C.c_uint))
        tileN, lenAX, lenSEC = (int(v) for v in out)
        ax, sec = np.zeros(lenAX, F64), np.zeros(lenSEC, U32)
        args = (C.c_uint(n), _p(row, C.c_uint), _p(col, C.c_uint), _p(val, C.c_double), _p(x, C.c_double))
        lg = 0
        if noc and th == 1:
            self.lib.orc_axt_fill_noc_h1(*args, C.c_uint(thw), _p(con, C.c_uint), _p(ax, C.c_double),
                                         _p(sec, C.c_uint))
        elif noc:
            self.lib.orc_axt_fill_noc(*args, C.c_uint(thw), C.c_uint(th), _p(con, C.c_uint), _p(ax, C.c_double),
                                      _p(sec, C.c_uint))
        else:
            lg = int(bs).bit_length() - 1
            self.lib.orc_axt_fill_com(*args, C.c_uint(thw), C.c_uint(bs), C.c_uint(lg), _p(ax, C.c_double),
                                      _p(sec, C.c_uint))
        return dict(con=con, ax=ax, sec=sec, tileN=tileN, lenAX=lenAX, lenSEC=lenSEC, log=lg)

    def axt_noc_h1_spmv(self, tileN, ax, sec, n):
        y = np.zeros(n, F64)
        self.lib.orc_axt_noc_h1_spmv(C.c_uint(tileN), _p(_d(ax), C.c_double), _p(_u(sec), C.c_uint),
                                     _p(y, C.c_double))
        return y

    def axt_noc_spmv(self, tileN, th, ax, sec, n):
        y = np.zeros(n, F64)
        self.lib.orc_axt_noc_spmv(C.c_uint(tileN), C.c_uint(th), _p(_d(ax), C.c_double), _p(_u(sec), C.c_uint),
                                  _p(y, C.c_double))
        return y

    def axt_com_h1_ref(self, bs, lg, tileN, lenSEC, ax, sec, n):
        y = np.zeros(n, F64)
        if self.lib.orc_axt_com_h1_ref(C.c_uint(bs), C.c_uint(lg), C.c_uint(tileN), C.c_uint(lenSEC),
                                       _p(_d(ax), C.c_double), _p(_u(sec), C.c_uint), _p(y, C.c_double)) != 0:
            raise MemoryError("orc_axt_com_h1_ref")
        return y


class Reference:
    """The reference (intSpmv_main.c) compiled from its own source."""

    @staticmethod
    def available() -> bool:
        if not REF_SO.exists():
            return False
        # the reference kernels are AVX-512
        try:
            with open("/proc/cpuinfo") as f:
                return "avx512f" in f.read()
        except OSError:
            return False

    def __init__(self):
        if not self.available():
            raise RuntimeError(f"reference library {REF_SO} unavailable")
        self.lib = C.CDLL(str(REF_SO))
        self.lib.ref_sizeof.restype = C.c_size_t
        self.lib.ref_time_kernel.restype = C.c_double
        self.lib.ref_k1p_mask_of.restype = C.c_uint
        self._libc = C.CDLL(None)
        self._libc.free.argtypes = [C.c_void_p]

    def sizeof(self, which: int) -> int:
        return int(self.lib.ref_sizeof(which))

    def num_ite(self) -> int:
        return int(self.lib.ref_num_ite())

    def csr(self, row, col, val):
        """A str_matCSR over numpy arrays (kept alive on the struct)."""
        row, col, val = _u(row), _u(col), _d(val)
        n = len(row) - 1
        s = abi.StrMatCSR()
        s.nrows, s.nnz = n, len(col)
        rl = np.zeros(n, U32)
        s.val, s.row, s.col, s.rl = _p(val, C.c_double), _p(row, C.c_uint), _p(col, C.c_uint), _p(rl, C.c_uint)
        s._keep = (row, col, val, rl)
        return s

    def stats(self, path: str, s):
        self.lib.ref_stats(str(path).encode(), C.byref(s))
        rl = s._keep[3]
        return dict(rl=rl.copy(), rmin=s.rmin, rave=s.rave, rmax=s.rmax, rsd=s.rsd, bw=s.bw)

    def free(self, *ptrs):
        for p in ptrs:
            if p:
                self._libc.free(C.cast(p, C.c_void_p))

    @staticmethod
    def _arr(ptr, n, dt):
        if n == 0:
            return np.zeros(0, dt)
        return np.ctypeslib.as_array(ptr, shape=(n,)).view(dt).copy()

    def build_axc(self, s, x, ompNT=1):
        x = _d(x)
        m, fd = abi.StrMatAXC(), abi.StrFormatData()
        self.lib.ref_build_axc(C.c_uint(ompNT), C.byref(s), _p(x, C.c_double), C.byref(m), C.byref(fd))
        out = dict(brp=self._arr(m.brp, m.lenBRP, U32), ax=self._arr(m.ax, m.lenAX, F64), lenAX=m.lenAX,
                   lenBRP=m.lenBRP, fd=(fd.name.decode(), fd.mfp, fd.beta), struct=m)
        return out

    def build_k1(self, s, x):
        x = _d(x)
        m, fd = abi.StrMatK1(), abi.StrFormatData()
        self.lib.ref_build_k1(C.byref(s), _p(x, C.c_double), C.byref(m), C.byref(fd))
        cn = m.chunkNum
        return dict(permi=self._arr(m.permi, (cn + 1) * 8, U32), nmc=self._arr(m.nmc, cn, U32),
                    chp=self._arr(m.chp, cn, U32), val=self._arr(m.val, m.lenVC, F64),
                    col=self._arr(m.col, m.lenVC, U32), chunkNum=cn, lenVC=m.lenVC,
                    fd=(fd.name.decode(), fd.mfp, fd.beta), struct=m)

    def build_axt(self, s, x, thw, th, mode, bs=128, ompNT=1):
        x = _d(x)
        m, fd = abi.StrMatAXT(), abi.StrFormatData()
        self.lib.ref_build_axt(C.c_uint(ompNT), C.c_uint(bs), C.c_uint(thw), C.c_uint(th), mode.encode(),
                               C.byref(s), _p(x, C.c_double), C.byref(m), C.byref(fd))
        return dict(con=self._arr(m.con, m.lenCON, U32), ax=self._arr(m.ax, m.lenAX, F64),
                    sec=self._arr(m.sec, m.lenSEC, U32), tileN=m.tileN, lenAX=m.lenAX, lenSEC=m.lenSEC,
                    lenCON=m.lenCON, log=m.log, logTH=m.logTH, mode=m.mode.decode(), tileHW=m.tileHW,
                    tileH=m.tileH, fd=(fd.name.decode(), fd.mfp, fd.beta), struct=m)

    def free_axc(self, d):
        m = d["struct"]
        self.free(m.ax, m.brp)

    def free_k1(self, d):
        m = d["struct"]
        self.free(m.permi, m.nmc, m.chp, m.val, m.col)

    def free_axt(self, d):
        m = d["struct"]
        self.free(m.ax, m.sec, m.con)

    def cf_csr(self, s, x):
        x = _d(x)
        y = np.zeros(s.nrows, F64)
        self.lib.ref_cf_csr(C.byref(s), _p(x, C.c_double), _p(y, C.c_double))
        return y

    def int_axc(self, d, n, ompNT=1):
        y = np.zeros(n, F64)
        self.lib.ref_int_axc(C.c_uint(ompNT), C.byref(d["struct"]), _p(y, C.c_double))
        return y

    def int_k1(self, d, x, n, ompNT=1):
        x = _d(x)
        res = np.zeros(d["chunkNum"] * 8, F64)
        y = np.zeros(n, F64)
        self.lib.ref_int_k1(C.c_uint(ompNT), C.byref(d["struct"]), _p(x, C.c_double), _p(res, C.c_double),
                            _p(y, C.c_double))
        return res, y

    def int_k1p(self, d, x, n, ompNT=1):
        x = _d(x)
        y = np.zeros(n + 1, F64)
        self.lib.ref_int_k1p(C.c_uint(ompNT), C.byref(d["struct"]), _p(x, C.c_double), _p(y, C.c_double))
        return y[:n]

    def int_axt(self, d, n, bs=128, ompNT=1):
        y = np.zeros(n, F64)
        m = d["struct"]
        if d["mode"] == "COM":
            self.lib.ref_int_axt_com_h1(C.c_uint(ompNT), C.c_uint(bs), C.byref(m), _p(y, C.c_double))
        elif d["tileH"] == 1:
            self.lib.ref_int_axt_noc_h1(C.c_uint(ompNT), C.byref(m), _p(y, C.c_double))
        else:
            self.lib.ref_int_axt_noc(C.c_uint(ompNT), C.byref(m), _p(y, C.c_double))
        return y

    def get_errors(self, ref, res):
        ref, res = _d(ref), _d(res)
        e = abi.StrErr()
        self.lib.ref_get_errors(C.c_uint(len(ref)), _p(ref, C.c_double), _p(res, C.c_double), C.byref(e))
        return e.aErr, e.rErr, e.pos

    KINDS = {"cf_CSR": 0, "int_axc": 1, "int_k1": 2, "int_k1p": 3, "int_axt_noc_h1": 4, "int_axt_noc": 5,
             "int_axt_com_h1": 6}

    def time_kernel(self, kind: str, mat, x, n, work_len=0, bs=0, iters=1, ompNT=None):
        """Seconds per call of a reference kernel (its own gettimeofday
        timing, as its test_* wrappers do).  Returns (et, ot)."""
        ompNT = ompNT or os.cpu_count() or 1
        x = _d(x)
        y = np.zeros(n + 1, F64)
        work = np.zeros(max(work_len, 1), F64)
        ot = C.c_double()
        et = self.lib.ref_time_kernel(C.c_int(self.KINDS[kind]), C.c_uint(ompNT), C.byref(mat), C.c_uint(bs),
                                      _p(x, C.c_double), _p(work, C.c_double), _p(y, C.c_double), C.c_int(iters),
                                      C.byref(ot))
        return et, ot.value, y[:n]
