"""Format conversion on the GPU (ispmv_dev_build_axt): the AXT arrays of
getFormatDataAXT built from device CSR arrays are bit-identical to the host
builder's (which the golden fixtures pin to the reference), for NOC at
tileHeight 1, 3, 4, 8, 16, 48 and COM at bs 8, 128, 256, 512; the
reference's kernels on them match the CSR oracle; and the multi-block prefix
scan is exercised past one block of block totals (> 4M rows)."""
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
