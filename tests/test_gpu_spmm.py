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


def check_spmm(env, row, col, val, fmt, kernel, k, val_kind="f64", seed=0):
    torch, D, F, orc = env
    n = len(row) - 1
    X = np.random.default_rng(seed).uniform(-1, 1, (n, k))
    csr = F.CSR(row, col, val)
    p = make_plan(F, D, csr, X[:, 0], fmt, kernel=kernel, val=val_kind)
    Y = torch.full((n, k), 9.0, dtype=torch.float64, device="cuda")
    p.spmm(torch.from_numpy(X).cuda(), Y)
    Yh = Y.cpu().numpy()
    tol = TOL_F64 if val_kind == "f64" else TOL_F32
    for j in range(k):
        xj = np.ascontiguousarray(X[:, j])
        assert_parity(Yh[:, j], orc.cf_csr(row, col, val, xj), orc.abs_csr(row, col, val, xj), tol,
                      what=f"{fmt} k={k} col {j}")


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("fmt,kernel", STREAM)
@pytest.mark.parametrize("k", [1, 8, 13, 32, 40])
def test_spmm_golden(env, name, fmt, kernel, k):
    g = load_golden(name)
    check_spmm(env, g["row"], g["col"], g["val"], fmt, kernel, k)


@pytest.mark.parametrize("fmt,kernel", STREAM)
@pytest.mark.parametrize("k", [8, 16, 32])
@pytest.mark.parametrize("val_kind", ["f64", "f32"])
def test_spmm_random(env, fmt, kernel, k, val_kind):
    from int_spmv_b200 import matrices as M
    row, col, val = M.random_csr(9000, 31, rl_max=120, empty_frac=0.1)
    check_spmm(env, row, col, val, fmt, kernel, k, val_kind)


@pytest.mark.parametrize("k,rhs_block", [(5, 8), (7, 16), (9, 8), (31, 32), (33, 16), (12, 32), (64, 32)])
def test_spmm_rhs_blocks_and_odd_k(env, k, rhs_block):
    """Every RHS block on k that is odd (scalar X loads and stores), not a
    multiple of the block (a partial last block), or several blocks."""
    torch, D, F, orc = env
    from int_spmv_b200 import matrices as M
    row, col, val = M.random_csr(7001, 13, rl_max=90, empty_frac=0.08)
    n = len(row) - 1
    X = np.random.default_rng(k).uniform(-1, 1, (n, k))
    csr = F.CSR(row, col, val)
    p = make_plan(F, D, csr, X[:, 0], "COM128", kernel="wide", rhs_block=rhs_block)
    Y = torch.full((n, k), 9.0, dtype=torch.float64, device="cuda")
    p.spmm(torch.from_numpy(X).cuda(), Y)
    Yh = Y.cpu().numpy()
    for j in range(k):
        xj = np.ascontiguousarray(X[:, j])
        assert_parity(Yh[:, j], orc.cf_csr(row, col, val, xj), orc.abs_csr(row, col, val, xj), TOL_F64,
                      what=f"k={k} block={rhs_block} col {j}")
    # X and Y 8 bytes into their buffers: no 16-byte vector access
    Xb = torch.zeros(n * k + 1, dtype=torch.float64, device="cuda")
    Xb[1:] = torch.from_numpy(X.reshape(-1)).cuda()
    Yb = torch.full((n * k + 1,), 9.0, dtype=torch.float64, device="cuda")
    p.spmm(Xb[1:].view(n, k), Yb[1:].view(n, k))
    assert np.array_equal(Yb[1:].view(n, k).cpu().numpy(), Yh)


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
