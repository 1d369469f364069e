"""Host builders at the benchmark scale, byte for byte against the
reference itself (intSpmv_main.c compiled from its own source into
oracle/_ref): the 2D Poisson 512x512 matrix (n = 262,144) and the power-law
matrix with n = 4,000,000 (lognormal(2.2, 1.0) row lengths, seed 1,
59,574,203 nonzeros).

Per format: AXC brp/ax (getFormatDataAXC, intSpmv_main.c:662-707), K1
permi/nmc/chp/val/col (getFormatDataK1, :841-905 - at 4M rows the row order
is the reference's qsort order, :775-796, through its many ties of equal row
length), and AXT con/sec/ax for the uncompacted layout at tileH 1, 4 and 8
and the compacted one at bs 128, 256 and 512 (getFormatDataAXT,
:1275-1381), plus each formats-table row (name, footprint, occupancy).
"""
from __future__ import annotations

import numpy as np
import pytest

from int_spmv_b200 import formats as F
from int_spmv_b200 import matrices as M
from oracle import Reference

pytestmark = pytest.mark.skipif(not Reference.available(), reason="oracle/_ref (the compiled reference) is absent")

AXT = [("NOC", 1, 128), ("NOC", 4, 128), ("NOC", 8, 128), ("COM", 1, 128), ("COM", 1, 256), ("COM", 1, 512)]


@pytest.fixture(scope="module", params=["poisson512", "powerlaw4m"])
def mat(request):
    if request.param == "poisson512":
        row, col, val = M.poisson2d(512)
        x = M.uniform_x(512 * 512, 0)
    else:
        row, col, val = M.powerlaw(4_000_000, seed=1)
        x = M.uniform_x(4_000_000, 1)
    R = Reference()
    s = R.csr(row, col, val)
    s._keep[3][:] = np.diff(row)  # rl, which the reference fills in its stats pass
    return request.param, F.CSR(row, col, val), x, R, s


def _same_fd(fd, ref_fd):
    name, mfp, beta = ref_fd
    assert fd.name == name and fd.mfp == mfp
    assert (np.isnan(fd.beta) and np.isnan(beta)) or fd.beta == beta, (fd.beta, beta)


def test_scale_sizes(mat):
    name, csr, *_ = mat
    assert (csr.n, csr.nnz) == {"poisson512": (262_144, 1_308_672), "powerlaw4m": (4_000_000, 59_574_203)}[name]


def test_scale_axc(mat):
    _, csr, x, R, s = mat
    fd, m = F.getFormatDataAXC(0, csr, x)
    d = R.build_axc(s, x, ompNT=8)
    try:
        assert np.array_equal(m.brp, d["brp"])
        assert np.array_equal(m.ax.view(np.uint64), d["ax"].view(np.uint64))
        _same_fd(fd, d["fd"])
    finally:
        R.free_axc(d)


def test_scale_k1(mat):
    _, csr, x, R, s = mat
    fd, m = F.getFormatDataK1(8, csr, x)
    d = R.build_k1(s, x)
    try:
        for f in ("permi", "nmc", "chp", "col"):
            assert np.array_equal(getattr(m, f), d[f]), f
        assert np.array_equal(m.val.view(np.uint64), d["val"].view(np.uint64))
        _same_fd(fd, d["fd"])
    finally:
        R.free_k1(d)


@pytest.mark.parametrize("mode,th,bs", AXT)
def test_scale_axt(mat, mode, th, bs):
    _, csr, x, R, s = mat
    fd, m = F.getFormatDataAXT(0, bs, 8, th, mode, csr, x)
    d = R.build_axt(s, x, 8, th, mode, bs, ompNT=8)
    try:
        assert np.array_equal(m.con, d["con"])
        assert np.array_equal(m.sec, d["sec"])
        assert np.array_equal(m.ax.view(np.uint64), d["ax"].view(np.uint64))
        assert (m.c.tileN, m.c.lenAX, m.c.lenSEC, m.c.lenCON) == (d["tileN"], d["lenAX"], d["lenSEC"], d["lenCON"])
        _same_fd(fd, d["fd"])
    finally:
        R.free_axt(d)
