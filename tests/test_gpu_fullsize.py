"""Full-size parity of the benchmark workloads that the plan tests cover only
at small sizes, every row against the oracle's CSR product
(|y_i - y_ref_i| <= tol (|A||x|)_i; tol 1e-12 for FP64 values, 1e-6 for
the FP32-value forms):

- the 3D 27-point stencil 160^3 (n = 4,096,000, nnz = 109,215,352; diagonal
  26, off-diagonal -1 + U[-0.1, 0.1], seed 2) in every value and column form:
  FP64, FP32 values, FP32 + BF16 lo-word, FP32 + 16-bit column deltas and
  FP64 + 16-bit column deltas, each on the kernel AUTO picks;
- multi-RHS SpMM on the power-law generator at n = 1,000,000 (seed 3), X
  n x k U[-1, 1] for k = 8, 16, 32, FP64 and FP32 values: every column;
- the 512 banded FEM-like matrices (n log-uniform in [1e3, 2e5], seed 4;
  21.7M rows, 956M nonzeros) as one block-diagonal plan in one CUDA-graph
  launch, each matrix against its own product.
"""
from __future__ import annotations

import numpy as np
import pytest

from paritylib import TOL_F32, TOL_F64, assert_parity

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch

    from int_spmv_b200 import device as D
    from int_spmv_b200 import formats as F
    from oracle import Oracle
    return torch, D, F, Oracle()


@pytest.fixture(scope="module")
def stencil160(env):
    torch, D, F, orc = env
    from int_spmv_b200 import matrices as M
    row, col, val = M.stencil27(160, seed=2)
    x = M.uniform_x(160 ** 3, 2)
    csr = F.CSR(row, col, val)
    com = F.getFormatDataAXT(0, 128, 8, 1, "COM", csr, x)[1]
    return csr, com, x, orc.cf_csr(row, col, val, x), orc.abs_csr(row, col, val, x)


@pytest.mark.parametrize("val_kind,col_kind", [("f64", "u32"), ("f32", "u32"), ("f32lo", "u32"), ("f32", "d16"),
                                               ("f64", "d16")])
def test_stencil160_forms(env, stencil160, val_kind, col_kind):
    torch, D, F, orc = env
    csr, com, x, yref, absax = stencil160
    assert (csr.n, csr.nnz) == (4_096_000, 109_215_352)
    p = D.Plan(csr, com, val=val_kind, col=col_kind)
    xt = torch.from_numpy(x).cuda()
    y = p.spmv(xt).cpu().numpy()
    assert p.status() == 0
    assert_parity(y, yref, absax, TOL_F64 if val_kind == "f64" else TOL_F32,
                  what=f"stencil 160^3 {val_kind}/{col_kind} {p.kernel_name()}")
    y2 = p.spmv(xt).cpu().numpy()
    assert np.array_equal(y, y2)  # bitwise repeatable
    del p


@pytest.fixture(scope="module")
def powerlaw1m(env):
    torch, D, F, orc = env
    from int_spmv_b200 import matrices as M
    row, col, val = M.powerlaw(1_000_000, seed=3)
    return row, col, val, F.CSR(row, col, val)


@pytest.mark.parametrize("k", [8, 16, 32])
@pytest.mark.parametrize("val_kind", ["f64", "f32"])
@pytest.mark.parametrize("fmt", ["COM128", "NOC1"])
@pytest.mark.parametrize("spmm_kernel", ["wide", "ldg"])
def test_spmm_powerlaw1m_every_column(env, powerlaw1m, fmt, val_kind, k, spmm_kernel):
    torch, D, F, orc = env
    from test_gpu_plan import make_plan
    row, col, val, csr = powerlaw1m
    n = csr.n
    X = np.random.default_rng(3).uniform(-1, 1, (n, k))
    p = make_plan(F, D, csr, X[:, 0], fmt, kernel="ldg", rhs_block=k, val=val_kind, spmm_kernel=spmm_kernel)
    Y = torch.full((n, k), 7.0, dtype=torch.float64, device="cuda")
    p.spmm(torch.from_numpy(X).cuda(), Y)
    Yh = Y.cpu().numpy()
    tol = TOL_F64 if val_kind == "f64" else TOL_F32
    for j in range(k):
        xj = np.ascontiguousarray(X[:, j])
        assert_parity(Yh[:, j], orc.cf_csr(row, col, val, xj), orc.abs_csr(row, col, val, xj), tol,
                      what=f"SpMM {fmt} {val_kind} k={k} column {j}")


@pytest.fixture(scope="module")
def fem512(env):
    torch, D, F, orc = env
    from int_spmv_b200 import batch as B
    from int_spmv_b200 import matrices as M
    mats = M.fem_batch_c(count=512, seed=4, n_lo=1e3, n_hi=2e5)
    big, off = B.blockdiag(mats)
    x = M.uniform_x(big.n, 4)
    refs = []
    for m, (row, col, val) in enumerate(mats):
        a, b = int(off[m]), int(off[m + 1])
        refs.append((orc.cf_csr(row, col, val, x[a:b]), orc.abs_csr(row, col, val, x[a:b])))
    del mats
    return big, off, x, refs


@pytest.mark.parametrize("val_kind,kw", [("f64", dict(kernel="wide")), ("f32", dict(kernel="wide")),
                                         ("f64", dict(kernel="ldg", variant=16))])
def test_fem512_one_graph_launch(env, fem512, val_kind, kw):
    torch, D, F, orc = env
    big, off, x, refs = fem512
    assert len(refs) == 512 and big.nnz > 9e8
    p = D.Plan(big, None, val=val_kind, **kw)
    xt = torch.from_numpy(x).cuda()
    y = torch.full((big.n,), 5.0, dtype=torch.float64, device="cuda")
    tol = TOL_F64 if val_kind == "f64" else TOL_F32
    for rep in range(2):  # the first call captures the graph, the second replays it
        y.fill_(5.0)
        p.spmv_graph(xt, y)
        yh = y.cpu().numpy()
        for m, (yref, absax) in enumerate(refs):
            a, b = int(off[m]), int(off[m + 1])
            assert_parity(yh[a:b], yref, absax, tol, what=f"fem batch {val_kind} {kw} matrix {m} rep {rep}")
    assert p.status() == 0
    del p
