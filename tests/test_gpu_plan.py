"""Plans (formats resident in HBM, fresh x per call) against the oracle's
CSR product: every format, FP64 and FP32 values, beta 0 and 1, the golden
edge cases, segment-boundary stress, determinism, end-to-end host calls, and
the two full-size workloads (Poisson 512^2; power-law n = 4M)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_names, load_golden
from paritylib import TOL_F32, TOL_F64, assert_parity

pytestmark = pytest.mark.gpu

FORMATS = ["CSR", "AXC", "K1", "K1P", "NOC1", "NOC4", "NOC8", "NOC16", "NOC3", "COM128", "COM256", "COM512"]


@pytest.fixture(scope="module")
def env():
    import torch
    from int_spmv_b200 import device as D
    from int_spmv_b200 import formats as F
    from oracle import Oracle
    return torch, D, F, Oracle()


def make_plan(F, D, csr, x, fmt, **kw):
    if fmt == "CSR":
        return D.Plan(csr, None, **kw)
    if fmt == "AXC":
        return D.Plan(csr, F.getFormatDataAXC(0, csr, x)[1], **kw)
    if fmt in ("K1", "K1P"):
        return D.Plan(csr, F.getFormatDataK1(8, csr, x)[1], reorder=fmt == "K1P", **kw)
    if fmt.startswith("NOC"):
        return D.Plan(csr, F.getFormatDataAXT(0, 128, 8, int(fmt[3:]), "NOC", csr, x)[1], **kw)
    if fmt.startswith("COM"):
        return D.Plan(csr, F.getFormatDataAXT(0, int(fmt[3:]), 8, 1, "COM", csr, x)[1], **kw)
    raise ValueError(fmt)


def check_plan(env, row, col, val, x, fmt, val_kind="f64", beta=0, **kw):
    torch, D, F, orc = env
    csr = F.CSR(row, col, val)
    p = make_plan(F, D, csr, x, fmt, val=val_kind, **kw)
    n = csr.n
    xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    y0 = np.random.default_rng(5).uniform(-1, 1, n)
    yt = torch.from_numpy(y0.copy()).cuda()
    p.spmv(xt, yt, beta=beta)
    y = yt.cpu().numpy()
    ref = orc.cf_csr(row, col, val, x) + (y0 if beta else 0.0)
    absax = orc.abs_csr(row, col, val, x) + (np.abs(y0) * 1e-4 if beta else 0.0)
    assert_parity(y, ref, absax, TOL_F64 if val_kind == "f64" else TOL_F32, what=f"{fmt}/{val_kind}/beta{beta}")
    return p, xt


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("fmt", FORMATS)
@pytest.mark.parametrize("val_kind", ["f64", "f32"])
def test_golden(env, name, fmt, val_kind):
    g = load_golden(name)
    for beta in (0, 1):
        check_plan(env, g["row"], g["col"], g["val"], g["x"], fmt, val_kind, beta)


@pytest.mark.parametrize("fmt", FORMATS)
def test_segment_boundaries(env, fmt):
    """Small warp segments and long rows: rows span many segments."""
    from int_spmv_b200 import matrices as M
    row, col, val = M.random_csr(3001, 9, rl_max=700, empty_frac=0.2)
    x = M.uniform_x(3001, 9)
    for upw in (32, 64, 0):
        check_plan(env, row, col, val, x, fmt, units_per_warp=upw)


@pytest.mark.parametrize("fmt", ["NOC1", "NOC4", "COM128", "CSR", "K1P"])
def test_deterministic_and_host_e2e(env, fmt):
    torch, D, F, orc = env
    from int_spmv_b200 import matrices as M
    row, col, val = M.random_csr(20000, 4, rl_max=60, empty_frac=0.05)
    x = M.uniform_x(20000, 4)
    p, xt = check_plan(env, row, col, val, x, fmt)
    a = p.spmv(xt).cpu().numpy()
    b = p.spmv(xt).cpu().numpy()
    assert np.array_equal(a, b)  # no atomics on the plan path: bitwise repeatable
    hx = torch.from_numpy(x.copy()).pin_memory()
    hy = torch.empty(20000, dtype=torch.float64).pin_memory()
    p.spmv_host(hx, hy)
    assert np.array_equal(hy.numpy(), a)


@pytest.fixture(scope="module")
def poisson512(env):
    from int_spmv_b200 import matrices as M
    row, col, val = M.poisson2d(512)
    return row, col, val, M.uniform_x(len(row) - 1, 0)


@pytest.mark.parametrize("fmt", ["CSR", "NOC1"])
def test_poisson512(env, poisson512, fmt):
    row, col, val, x = poisson512
    assert len(row) - 1 == 262144 and len(col) == 1308672
    check_plan(env, row, col, val, x, fmt)


@pytest.fixture(scope="module")
def powerlaw4m(env):
    from int_spmv_b200 import matrices as M
    row, col, val = M.powerlaw(4_000_000, seed=1)
    return row, col, val, M.uniform_x(4_000_000, 1)


@pytest.mark.parametrize("fmt", ["CSR", "AXC", "K1P", "NOC1", "NOC4", "NOC8", "COM128", "COM512"])
def test_powerlaw_4m(env, powerlaw4m, fmt):
    row, col, val, x = powerlaw4m
    check_plan(env, row, col, val, x, fmt)
    if fmt in ("COM128", "NOC1"):
        check_plan(env, row, col, val, x, fmt, val_kind="f32")
