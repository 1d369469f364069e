"""Plans built on the GPU from a device CSR (ispmv_plan_dev_csr): every
array of the plan (lane-interleaved values and columns, row-start bitmap,
segment start counts, row map, empty-row list) is bit-identical to the plan
ispmv_plan_csr builds on the host from the same matrix and variant; the
products of both plans are bitwise equal and match the CSR oracle; and a
malformed CSR is rejected before any kernel indexes through it."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_names, load_golden
from paritylib import TOL_F32, TOL_F64, assert_parity

pytestmark = pytest.mark.gpu

# plain-load (4: 8 slots/lane; 0, 9: 16 slots/lane), bulk-copy staged (11), per-CTA x
# window (26) and column prefetch (32) variants
VARIANTS = [4, 0, 9, 11, 26, 32]


def _dev(a):
    from int_spmv_b200 import device as D
    return D.to_device(np.ascontiguousarray(a))


def check_dev_plan(row, col, val, x, val_kind, variant, units_per_warp=0, kernel="wide"):
    import torch

    from int_spmv_b200 import device as D
    from int_spmv_b200 import formats as F
    from oracle import Oracle
    n = len(row) - 1
    dcol = _dev(col if len(col) else np.zeros(1, np.uint32))
    dval = _dev(val if len(val) else np.zeros(1))
    pd = D.Plan.from_device_csr(_dev(row), dcol[:len(col)], dval[:len(val)], val_kind=val_kind, kernel=kernel,
                                variant=variant, units_per_warp=units_per_warp)
    chosen = pd.info
    ph = D.Plan(F.CSR(row, col, val), None, kernel="wide", variant=variant if variant else 0, val=val_kind,
                units_per_warp=units_per_warp) if kernel == "wide" else None
    a = pd.export_stream()
    if ph is not None:
        b = ph.export_stream()
        assert a["layout"] == b["layout"]
        for k in ("val", "col", "heads", "segh", "rowmap", "empty", "win_lo", "win_len"):
            assert np.array_equal(a[k], b[k]), k
        assert chosen["device_bytes"] == ph.info["device_bytes"]
        assert chosen["alg_bytes"] == ph.info["alg_bytes"]
    xt = torch.from_numpy(x).cuda()
    y = pd.spmv(xt).cpu().numpy()
    orc = Oracle()
    assert_parity(y, orc.cf_csr(row, col, val, x), orc.abs_csr(row, col, val, x),
                  TOL_F64 if val_kind == "f64" else TOL_F32, what=f"dev plan v{variant}/{val_kind}")
    if ph is not None:
        assert np.array_equal(y.view(np.uint64), ph.spmv(xt).cpu().numpy().view(np.uint64))
    assert pd.status() == 0
    return pd


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("val_kind", ["f64", "f32"])
def test_dev_plan_matches_host_golden(name, variant, val_kind):
    g = load_golden(name)
    check_dev_plan(g["row"], g["col"], g["val"], g["x"], val_kind, variant)


@pytest.mark.parametrize("variant", VARIANTS)
def test_dev_plan_random_and_segments(variant):
    """Random rows with empty ones, rows longer than a segment, small warp
    segments, and a power-law matrix of 200,003 rows."""
    from int_spmv_b200 import matrices as M
    mats = [M.random_csr(7001, 12, rl_max=90, empty_frac=0.1), M.random_csr(3001, 9, rl_max=700, empty_frac=0.2),
            M.powerlaw(200_003, seed=4)]
    for i, (row, col, val) in enumerate(mats):
        x = M.uniform_x(len(row) - 1, 20 + i)
        for upw in (0, 64):
            check_dev_plan(row, col, val, x, "f64", variant, units_per_warp=upw)


@pytest.mark.parametrize("val_kind", ["f64", "f32"])
def test_dev_plan_auto_picks_the_compacted_default(val_kind):
    """kernel=auto picks the kernel ispmv_plan_axt picks for the compacted
    AXT of the same matrix, the scatter test run on the device: short
    scattered rows (per-CTA window / column prefetch), short rows on fixed
    far diagonals, long structured rows (bulk-copy staged for FP64) and long
    scattered rows."""
    import torch

    from int_spmv_b200 import device as D
    from int_spmv_b200 import formats as F
    from int_spmv_b200 import matrices as M
    n = 20000
    r = np.repeat(np.arange(n), 3)
    c = (r + np.tile([-1700, 0, 1700], n)) % n
    order = np.lexsort((c, r))
    diag = (np.arange(0, 3 * n + 1, 3, dtype=np.uint32), c[order].astype(np.uint32),
            np.random.default_rng(2).normal(size=3 * n))
    mats = [M.random_csr(5001, 3, rl_max=20, empty_frac=0.05), diag, M.stencil27(20, seed=2),
            M.random_csr(6001, 5, rl_max=60, empty_frac=0.05)]
    for row, col, val in mats:
        x = M.uniform_x(len(row) - 1, 3)
        pd = check_dev_plan(row, col, val, x, val_kind, 0, kernel="auto")
        csr = F.CSR(row, col, val)
        ph = D.Plan(csr, F.getFormatDataAXT(0, 128, 8, 1, "COM", csr, x)[1], val=val_kind)
        xt = torch.from_numpy(x).cuda()
        pd.spmv(xt)
        ph.spmv(xt)
        assert pd.kernel_name() == ph.kernel_name(), (pd.kernel_name(), ph.kernel_name())


def test_dev_plan_rejects_malformed_and_unsupported():
    from int_spmv_b200 import abi
    from int_spmv_b200 import device as D
    from int_spmv_b200 import matrices as M
    from int_spmv_b200._lib import IntSpmvError
    row, col, val = M.random_csr(1001, 5, rl_max=30, empty_frac=0.1)
    bad_col = col.copy()
    bad_col[len(col) // 2] = 1001  # column == n
    bad_row = row.copy()
    bad_row[500] = bad_row[502] + 1  # decreasing pointer
    for r, c in ((row, bad_col), (bad_row, col)):
        with pytest.raises(IntSpmvError) as e:
            D.Plan.from_device_csr(_dev(r), _dev(c), _dev(val), kernel="wide", variant=4)
        assert e.value.status == abi.ERR_ARG
    for kw in (dict(kernel="wide", variant=22), dict(kernel="wide", variant=19), dict(kernel="ldg"),
               dict(val_kind="f32lo")):
        with pytest.raises(IntSpmvError) as e:
            D.Plan.from_device_csr(_dev(row), _dev(col), _dev(val), **kw)
        assert e.value.status == abi.ERR_UNSUPPORTED
