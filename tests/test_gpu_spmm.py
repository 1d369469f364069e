"""Multi-RHS SpMM (Y = A X, X and Y row-major n x k) on the slot-stream
plans, column by column against the oracle's CSR product."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_names, load_golden
from paritylib import TOL_F32, TOL_F64, assert_parity
from test_gpu_plan import make_plan

pytestmark = pytest.mark.gpu

STREAM = [("COM128", "ldg"), ("NOC1", "ldg"), ("AXC", "ldg"), ("CSR", "ldg"), ("COM512", "tma"), ("COM128", "wide"),
          ("NOC1", "wide"), ("COM256", "auto"), ("NOC4", "auto"), ("CSR", "auto")]


@pytest.fixture(scope="module")
def env():
    import torch

    from int_spmv_b200 import device as D
    from int_spmv_b200 import formats as F
    from oracle import Oracle
    return torch, D, F, Oracle()


def four_wide(spmm_kernel, k, rhs_block=0):
    """Whether ispmv_plan_spmm runs the four-columns-per-lane kernel
    (stream_spmm4) on an X from torch (32-byte aligned): "wide" always (k a
    multiple of 4), "auto" for blocks of 16 or 32 columns, "ldg" never."""
    block = rhs_block if rhs_block in (8, 16, 32) else (8 if k <= 8 else 16 if k <= 16 else 32)
    return k % 4 == 0 and (spmm_kernel == "wide" or (spmm_kernel == "auto" and block > 8))


def check_spmm(env, row, col, val, fmt, kernel, k, val_kind="f64", seed=0, spmm_kernel="auto"):
    torch, D, F, orc = env
    n = len(row) - 1
    X = np.random.default_rng(seed).uniform(-1, 1, (n, k))
    csr = F.CSR(row, col, val)
    p = make_plan(F, D, csr, X[:, 0], fmt, kernel=kernel, val=val_kind, spmm_kernel=spmm_kernel)
    Y = torch.full((n, k), 9.0, dtype=torch.float64, device="cuda")
    p.spmm(torch.from_numpy(X).cuda(), Y)
    assert p.kernel_name() == ("stream_spmm4" if four_wide(spmm_kernel, k) else "stream_spmm"), p.kernel_name()
    Yh = Y.cpu().numpy()
    tol = TOL_F64 if val_kind == "f64" else TOL_F32
    for j in range(k):
        xj = np.ascontiguousarray(X[:, j])
        assert_parity(Yh[:, j], orc.cf_csr(row, col, val, xj), orc.abs_csr(row, col, val, xj), tol,
                      what=f"{fmt} k={k} col {j}")


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("fmt,kernel", STREAM)
@pytest.mark.parametrize("k", [1, 8, 13, 32, 40])
@pytest.mark.parametrize("spmm_kernel", ["auto", "ldg", "wide"])
def test_spmm_golden(env, name, fmt, kernel, k, spmm_kernel):
    if k % 2 and spmm_kernel == "ldg":
        pytest.skip("odd k runs the two-column form under auto already")
    if k % 4 and spmm_kernel == "wide":
        pytest.skip("four columns per lane need k a multiple of 4")
    g = load_golden(name)
    check_spmm(env, g["row"], g["col"], g["val"], fmt, kernel, k, spmm_kernel=spmm_kernel)


@pytest.mark.parametrize("fmt,kernel", STREAM)
@pytest.mark.parametrize("k", [8, 16, 32])
@pytest.mark.parametrize("val_kind", ["f64", "f32"])
@pytest.mark.parametrize("spmm_kernel", ["auto", "ldg", "wide"])
def test_spmm_random(env, fmt, kernel, k, val_kind, spmm_kernel):
    from int_spmv_b200 import matrices as M
    row, col, val = M.random_csr(9000, 31, rl_max=120, empty_frac=0.1)
    check_spmm(env, row, col, val, fmt, kernel, k, val_kind, spmm_kernel=spmm_kernel)


@pytest.mark.parametrize("k,rhs_block", [(5, 8), (7, 16), (9, 8), (31, 32), (33, 16), (12, 32), (64, 32), (24, 16),
                                         (10, 8), (2, 32)])
@pytest.mark.parametrize("spmm_kernel", ["auto", "ldg", "wide"])
def test_spmm_rhs_blocks_and_odd_k(env, k, rhs_block, spmm_kernel):
    """Every RHS block on k that is odd (scalar X loads and stores), not a
    multiple of the block (a partial last block), or several blocks."""
    torch, D, F, orc = env
    from int_spmv_b200 import IntSpmvError
    from int_spmv_b200 import matrices as M
    if k % 4 and spmm_kernel == "wide":
        pytest.skip("four columns per lane need k a multiple of 4")
    row, col, val = M.random_csr(7001, 13, rl_max=90, empty_frac=0.08)
    n = len(row) - 1
    X = np.random.default_rng(k).uniform(-1, 1, (n, k))
    csr = F.CSR(row, col, val)
    p = make_plan(F, D, csr, X[:, 0], "COM128", kernel="wide", rhs_block=rhs_block, spmm_kernel=spmm_kernel)
    Y = torch.full((n, k), 9.0, dtype=torch.float64, device="cuda")
    p.spmm(torch.from_numpy(X).cuda(), Y)
    wide = p.kernel_name() == "stream_spmm4"
    assert wide == four_wide(spmm_kernel, k, rhs_block)
    Yh = Y.cpu().numpy()
    for j in range(k):
        xj = np.ascontiguousarray(X[:, j])
        assert_parity(Yh[:, j], orc.cf_csr(row, col, val, xj), orc.abs_csr(row, col, val, xj), TOL_F64,
                      what=f"k={k} block={rhs_block} col {j}")
    # X and Y 8 bytes into their buffers: no 16-byte vector access, and the
    # two-column form (four columns per lane need X 32-byte aligned)
    Xb = torch.zeros(n * k + 1, dtype=torch.float64, device="cuda")
    Xb[1:] = torch.from_numpy(X.reshape(-1)).cuda()
    Yb = torch.full((n * k + 1,), 9.0, dtype=torch.float64, device="cuda")
    if spmm_kernel == "wide":
        with pytest.raises(IntSpmvError):
            p.spmm(Xb[1:].view(n, k), Yb[1:].view(n, k))
        return
    p.spmm(Xb[1:].view(n, k), Yb[1:].view(n, k))
    assert p.kernel_name() == "stream_spmm"
    Ym = Yb[1:].view(n, k).cpu().numpy()
    if not wide:
        assert np.array_equal(Ym, Yh)
    for j in range(k):
        xj = np.ascontiguousarray(X[:, j])
        assert_parity(Ym[:, j], orc.cf_csr(row, col, val, xj), orc.abs_csr(row, col, val, xj), TOL_F64,
                      what=f"misaligned k={k} block={rhs_block} col {j}")


def test_spmm_wide_repeatable_and_rejects(env):
    """The four-column form gives the same bits on every run, and a plan
    that asks for it explicitly rejects k not a multiple of 4 and an X or Y
    that is not 32-byte aligned (AUTO then runs the two-column form)."""
    torch, D, F, orc = env
    from int_spmv_b200 import IntSpmvError
    from int_spmv_b200 import matrices as M
    row, col, val = M.random_csr(5003, 17, rl_max=200, empty_frac=0.05)
    n = len(row) - 1
    csr = F.CSR(row, col, val)
    Xh = np.random.default_rng(1).uniform(-1, 1, (n, 32))
    X = torch.from_numpy(Xh).cuda()
    p = make_plan(F, D, csr, Xh[:, 0], "COM128", kernel="wide", spmm_kernel="wide")
    Y1, Y2 = p.spmm(X), p.spmm(X)
    assert p.kernel_name() == "stream_spmm4"
    assert torch.equal(Y1, Y2)
    Yb = torch.full((n * 32 + 1,), 9.0, dtype=torch.float64, device="cuda")
    with pytest.raises(IntSpmvError):
        p.spmm(X, Yb[1:].view(n, 32))  # Y 8 bytes into its buffer
    pa = make_plan(F, D, csr, Xh[:, 0], "COM128", kernel="wide")
    pa.spmm(X, Yb[1:].view(n, 32))
    assert pa.kernel_name() == "stream_spmm"
    assert torch.allclose(Yb[1:].view(n, 32), Y1, rtol=0, atol=1e-12)
    for j in range(32):
        xj = np.ascontiguousarray(Xh[:, j])
        assert_parity(Y1[:, j].cpu().numpy(), orc.cf_csr(row, col, val, xj), orc.abs_csr(row, col, val, xj),
                      TOL_F64, what=f"wide col {j}")
    for kk in (6, 7, 2):
        with pytest.raises(IntSpmvError):
            p.spmm(torch.zeros((n, kk), dtype=torch.float64, device="cuda"))
    Xb = torch.zeros(n * 32 + 2, dtype=torch.float64, device="cuda")
    for off in (1, 2):  # 8 and 16 bytes into the buffer
        with pytest.raises(IntSpmvError):
            p.spmm(Xb[off:off + n * 32].view(n, 32))


def test_spmm_unsupported(env):
    torch, D, F, orc = env
    from int_spmv_b200 import IntSpmvError
    g = load_golden("random257_empty")
    csr = F.CSR(g["row"], g["col"], g["val"])
    X = torch.zeros((257, 8), dtype=torch.float64, device="cuda")
    for fmt, kw in (("K1P", {}), ("NOC4", {"kernel": "ldg"}), ("CSR", {"kernel": "rows"})):
        p = make_plan(F, D, csr, g["x"], fmt, **kw)
        with pytest.raises(IntSpmvError):
            p.spmm(X)
