"""Product host builders (libintspmv.so) against the reference's arrays:
bit-exact pointer, index, reorder and value arrays, the same struct fields
and formats-table rows (name, memory footprint, occupancy)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_names, load_golden
from int_spmv_b200 import IntSpmvError
from int_spmv_b200 import formats as F
from int_spmv_b200 import matrices as M
from oracle import Oracle

AXT_CASES = [("NOC", 1, 128), ("NOC", 4, 128), ("NOC", 8, 128), ("NOC", 16, 128), ("NOC", 48, 128), ("NOC", 3, 128),
             ("COM", 1, 128), ("COM", 1, 256), ("COM", 1, 512), ("COM", 1, 8)]


def _csr(g):
    return F.CSR(g["row"], g["col"], g["val"])


def _same_fd(fd, name, expect):
    """Formats-table row: the name, the memory footprint and the occupancy
    (beta, NaN in both when the format holds no slot), exactly."""
    mfp, beta = (float(v) for v in expect)
    assert fd.name == name
    assert fd.mfp == mfp
    assert (np.isnan(fd.beta) and np.isnan(beta)) or fd.beta == beta, (fd.beta, beta)


@pytest.mark.parametrize("name", golden_names())
def test_stats(name):
    g = load_golden(name)
    c = _csr(g)
    assert np.array_equal(c.rl[:c.n], g["rl"])
    s = c.stats()
    assert [s["rmin"], s["rave"], s["rmax"], s["rsd"], s["bw"]] == list(g["stats"])


@pytest.mark.parametrize("name", golden_names())
def test_axc(name):
    g = load_golden(name)
    c = _csr(g)
    fd, m = F.getFormatDataAXC(0, c, g["x"])
    assert np.array_equal(m.brp, g["axc_brp"]) and np.array_equal(m.ax, g["axc_ax"])
    _same_fd(fd, "AXC", g["axc_fd"])
    # column companion: every value slot's column, 0 on padding
    axi = m.cols()
    v = m.ax.reshape(-1, 16)[:, :8].reshape(-1)
    xc = m.ax.reshape(-1, 16)[:, 8:].reshape(-1)
    assert np.array_equal(g["x"][axi][v != 0], xc[v != 0])
    assert np.all(axi[v == 0][xc[v == 0] == 0] >= 0)


@pytest.mark.parametrize("name", golden_names())
def test_k1(name):
    g = load_golden(name)
    c = _csr(g)
    fd, m = F.getFormatDataK1(8, c, g["x"])
    for f in ("permi", "nmc", "chp", "val", "col"):
        assert np.array_equal(getattr(m, f), g["k1_" + f]), f
    _same_fd(fd, "K1", g["k1_fd"])
    assert m.mask == int(g["k1_mask"])


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("mode,th,bs", AXT_CASES)
def test_axt(name, mode, th, bs):
    g = load_golden(name)
    c = _csr(g)
    fd, m = F.getFormatDataAXT(0, bs, 8, th, mode, c, g["x"])
    key = f"axt_{mode}_{th}_{bs}"
    assert np.array_equal(m.con, g[key + "_con"])
    assert np.array_equal(m.ax, g[key + "_ax"])
    assert np.array_equal(m.sec, g[key + "_sec"])
    tileN, lenAX, lenSEC, lenCON, log, logTH = (int(v) for v in g[key + "_meta"])
    assert (m.c.tileN, m.c.lenAX, m.c.lenSEC, m.c.lenCON, m.c.logTH) == (tileN, lenAX, lenSEC, lenCON, logTH)
    if mode == "COM":
        assert m.c.log == log
    _same_fd(fd, str(g[key + "_name"]), g[key + "_fd"])
    # companion columns agree with the x copies wherever x is distinct per column
    axi = m.cols()
    v = m.ax.reshape(-1, 16)[:, :8].reshape(-1)
    xc = m.ax.reshape(-1, 16)[:, 8:].reshape(-1)
    live = v != 0
    assert np.array_equal(g["x"][axi[live]], xc[live])


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_builders_match_oracle_random(seed):
    """Larger random matrices (threaded builders) against the oracle."""
    orc = Oracle()
    row, col, val = M.random_csr(5001, seed, rl_max=120, empty_frac=0.07)
    x = M.uniform_x(5001, seed)
    c = F.CSR(row, col, val)
    rl = c.rl[:c.n]
    for mode, th, bs in AXT_CASES:
        _, m = F.getFormatDataAXT(4, bs, 8, th, mode, c, x)
        o = orc.axt(row, col, val, x, rl, 8, th, mode, bs)
        for f in ("con", "ax", "sec"):
            assert np.array_equal(getattr(m, f), o[f]), (mode, th, bs, f)
    _, k = F.getFormatDataK1(8, c, x)
    ok = orc.k1(row, col, val, rl)
    for f in ("permi", "nmc", "chp", "val", "col"):
        assert np.array_equal(getattr(k, f), ok[f])
    _, a = F.getFormatDataAXC(4, c, x)
    oa = orc.axc(row, col, val, x, rl)
    assert np.array_equal(a.brp, oa["brp"]) and np.array_equal(a.ax, oa["ax"])


def test_builder_errors():
    row, col, val = M.random_csr(50, 3, rl_max=10)
    c = F.CSR(row, col, val)
    x = M.uniform_x(50, 0)
    with pytest.raises(IntSpmvError):
        F.getFormatDataAXT(0, 128, 8, 4, "COM", c, x)  # COM with tileH > 1: unimplemented in the reference
    with pytest.raises(IntSpmvError):
        F.getFormatDataAXT(0, 100, 8, 1, "COM", c, x)  # block size not a power of two
    with pytest.raises(IntSpmvError):
        F.getFormatDataAXT(0, 128, 8, 1, "XYZ", c, x)
    with pytest.raises(IntSpmvError):
        F.getFormatDataAXT(0, 128, 8, 0, "NOC", c, x)
    bad = row.copy()
    bad[3], bad[4] = bad[4], bad[3] + 1  # non-monotone row pointers
    with pytest.raises(IntSpmvError):
        F.CSR(bad, col, val)
    badcol = col.copy()
    badcol[0] = 50  # column out of range
    with pytest.raises(IntSpmvError):
        F.CSR(row, badcol, val)


def test_com_row_overflow_rejected():
    """(row << log2 bs) must fit 32 bits (the reference silently wraps)."""
    n = (1 << 23) + 1
    row = np.zeros(n + 1, np.uint32)
    row[-1] = 1
    row[n] = 1
    c = F.CSR(row, np.array([n - 1], np.uint32), np.array([1.0]))
    x = np.zeros(n)
    with pytest.raises(IntSpmvError):
        F.getFormatDataAXT(0, 512, 8, 1, "COM", c, x)
    F.getFormatDataAXT(0, 256, 8, 1, "COM", c, x)  # 2^24 rows fit at bs 256


def test_errors_and_initvec():
    v = F.initVec(7)
    assert list(v) == list(range(7))
    ref = np.array([1.0, -2.0, 3.0])
    res = np.array([1.0, 2.5, -3.0])  # sign errors are invisible to the reference metric
    a, r, p = F.getErrors(ref, res)
    assert (a, p) == (0.5, 1) and r == 0.5 / 3.0


def test_blockdiag_host():
    from int_spmv_b200 import batch as B
    mats = [M.random_csr(n, s, rl_max=12, empty_frac=0.1) for n, s in ((50, 1), (7, 2), (300, 3))]
    big, off = B.blockdiag(mats)
    assert list(off) == [0, 50, 57, 357]
    assert big.n == 357 and big.nnz == sum(len(c) for _, c, _ in mats)
    for m, (row, col, val) in enumerate(mats):
        a = int(off[m])
        r0 = int(big.row[a])
        assert np.array_equal(big.col[r0:r0 + len(col)], col.astype(np.int64) + a)
        assert np.array_equal(big.val[r0:r0 + len(val)], val)
