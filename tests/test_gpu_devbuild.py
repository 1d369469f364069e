"""Format conversion on the GPU (ispmv_dev_build_axt, ispmv_dev_build_k1):
the AXT and K1 arrays built from device CSR arrays are bit-identical to the
host builders' (which the golden fixtures pin to the reference), for NOC at
tileHeight 1, 3, 4, 8, 16, 48, COM at bs 8, 128, 256, 512, and K1 with many
equal row lengths (the stable order); the reference's kernels on them match
the CSR oracle; and the multi-block prefix scan is exercised past one block
of block totals (> 4M rows)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_names, load_golden
from paritylib import TOL_F64, assert_parity

pytestmark = pytest.mark.gpu

SHAPES = [("NOC", 1, 128), ("NOC", 3, 128), ("NOC", 4, 128), ("NOC", 8, 128), ("NOC", 16, 128), ("NOC", 48, 128),
          ("COM", 1, 8), ("COM", 1, 128), ("COM", 1, 256), ("COM", 1, 512)]


def _dev(a):
    from int_spmv_b200 import device as D
    return D.to_device(np.ascontiguousarray(a))


def check_build(row, col, val, x, mode, th, bs, run_kernel=True):
    import torch

    from int_spmv_b200 import device as D
    from int_spmv_b200 import formats as F
    from oracle import Oracle
    csr = F.CSR(row, col, val)
    fd_h, h = F.getFormatDataAXT(0, bs, 8, th, mode, csr, x)
    d = D.DeviceAXT(_dev(row), _dev(col if len(col) else np.zeros(1, np.uint32)), _dev(val if len(val) else np.zeros(1)),
                    _dev(x), bs=bs, th=th, mode=mode)
    for f in ("tileN", "lenAX", "lenSEC", "lenCON", "log", "logTH", "tileH", "tileHW"):
        assert getattr(d.c, f) == getattr(h.c, f), f
    arrs = d.to_host()
    assert np.array_equal(arrs["con"], h.con)
    assert np.array_equal(arrs["sec"], h.sec)
    assert np.array_equal(arrs["ax"].view(np.uint64), h.ax.view(np.uint64))  # bit for bit
    assert d.fd.name.decode() == fd_h.name
    assert d.fd.mfp == fd_h.mfp and d.fd.beta == fd_h.beta
    assert d.conversion_s > 0
    if run_kernel:
        # the reference kernels on the device-built arrays; the compacted one
        # is judged against the CSR oracle (the reference's own result drops
        # row-0 segments, README.md:33)
        y = torch.zeros(csr.n, dtype=torch.float64, device="cuda")
        d.spmv(y)
        orc = Oracle()
        assert_parity(y.cpu().numpy(), orc.cf_csr(row, col, val, x), orc.abs_csr(row, col, val, x), TOL_F64,
                      what=f"{mode}{th}/{bs}")
    return d


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("mode,th,bs", SHAPES)
def test_device_axt_matches_host_golden(name, mode, th, bs):
    g = load_golden(name)
    check_build(g["row"], g["col"], g["val"], g["x"], mode, th, bs)


@pytest.mark.parametrize("mode,th,bs", SHAPES)
def test_device_axt_random(mode, th, bs):
    from int_spmv_b200 import matrices as M
    row, col, val = M.random_csr(30011, 41, rl_max=300, empty_frac=0.1)
    check_build(row, col, val, M.uniform_x(30011, 41), mode, th, bs)


def test_device_axt_many_rows():
    """n + 1 > 1024 scan blocks of 4096 entries: the block totals take more
    than one pass of the totals scan."""
    rng = np.random.default_rng(7)
    n = 4_300_000
    rl = rng.integers(0, 3, n)
    row = np.concatenate([[0], np.cumsum(rl)]).astype(np.uint32)
    rows = np.repeat(np.arange(n), rl)
    col = ((rows + rng.integers(0, 50, len(rows))) % n).astype(np.uint32)
    # distinct ascending columns within each row
    key = rows.astype(np.int64) * n + col
    key = np.unique(key)
    rows, col = (key // n).astype(np.int64), (key % n).astype(np.uint32)
    rl = np.bincount(rows, minlength=n)
    row = np.concatenate([[0], np.cumsum(rl)]).astype(np.uint32)
    val = rng.standard_normal(len(col))
    x = rng.uniform(-1, 1, n)
    for mode, th, bs in (("COM", 1, 128), ("NOC", 1, 128), ("NOC", 4, 128)):
        check_build(row, col, val, x, mode, th, bs, run_kernel=False)


def check_build_k1(row, col, val, x):
    import torch

    from int_spmv_b200 import device as D
    from int_spmv_b200 import formats as F
    from oracle import Oracle
    csr = F.CSR(row, col, val)
    fd_h, h = F.getFormatDataK1(8, csr, x)
    d = D.DeviceK1(_dev(row), _dev(col if len(col) else np.zeros(1, np.uint32)),
                   _dev(val if len(val) else np.zeros(1)))
    assert (d.c.chunkNum, d.c.lenVC, d.c.nrows, d.c.nnz) == (h.c.chunkNum, h.c.lenVC, h.c.nrows, h.c.nnz)
    a = d.to_host()
    assert np.array_equal(a["permi"], h.permi)
    assert np.array_equal(a["nmc"], h.nmc) and np.array_equal(a["chp"], h.chp)
    assert np.array_equal(a["col"], h.col)
    assert np.array_equal(a["val"].view(np.uint64), h.val.view(np.uint64))
    assert d.fd.name.decode() == fd_h.name and d.fd.mfp == fd_h.mfp and d.fd.beta == fd_h.beta
    xt = _dev(x)
    y = torch.zeros(csr.n + 8, dtype=torch.float64, device="cuda")
    d.spmv(xt, y)
    orc = Oracle()
    assert_parity(y[:csr.n].cpu().numpy(), orc.cf_csr(row, col, val, x), orc.abs_csr(row, col, val, x), TOL_F64,
                  what="K1 built on the GPU")


@pytest.mark.parametrize("name", golden_names())
def test_device_k1_matches_host_golden(name):
    g = load_golden(name)
    check_build_k1(g["row"], g["col"], g["val"], g["x"])


def test_device_k1_random_and_ties():
    from int_spmv_b200 import matrices as M
    for n, seed, rl_max in ((30011, 41, 300), (20000, 7, 3), (4099, 3, 64)):  # many equal lengths
        row, col, val = M.random_csr(n, seed, rl_max=rl_max, empty_frac=0.1)
        check_build_k1(row, col, val, M.uniform_x(n, seed))
