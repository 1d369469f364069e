"""Batched SpMV: many uneven FEM-like banded matrices as one block-diagonal
plan (work-queue kernel, one CUDA-graph launch) against each matrix's own
oracle product, and against per-matrix plans."""
from __future__ import annotations

import numpy as np
import pytest

from paritylib import TOL_F32, TOL_F64, assert_parity

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch_env():
    import torch

    from int_spmv_b200 import batch as B
    from int_spmv_b200 import device as D
    from int_spmv_b200 import formats as F
    from int_spmv_b200 import matrices as M
    from oracle import Oracle
    mats = M.fem_batch(count=24, seed=4, n_lo=1e3, n_hi=2e4)
    big, off = B.blockdiag(mats)
    x = M.uniform_x(big.n, 4)
    return torch, D, F, Oracle(), mats, big, off, x


@pytest.mark.parametrize("fmt", ["COM128", "NOC1"])
@pytest.mark.parametrize("variant", [16, 0])
@pytest.mark.parametrize("val_kind", ["f64", "f32"])
def test_batch_graph_matches_each_matrix(batch_env, fmt, variant, val_kind):
    torch, D, F, orc, mats, big, off, x = batch_env
    if fmt == "COM128":
        _, f = F.getFormatDataAXT(0, 128, 8, 1, "COM", big, x)
    else:
        _, f = F.getFormatDataAXT(0, 128, 8, 1, "NOC", big, x)
    p = D.Plan(big, f, kernel="ldg", variant=variant, val=val_kind)
    xt = torch.from_numpy(x).cuda()
    y = torch.empty(big.n, dtype=torch.float64, device="cuda")
    for rep in range(3):  # the captured graph replays
        y.fill_(5.0)
        p.spmv_graph(xt, y)
        yh = y.cpu().numpy()
        for m, (row, col, val) in enumerate(mats):
            a, b = int(off[m]), int(off[m + 1])
            xm = x[a:b]
            assert_parity(yh[a:b], orc.cf_csr(row, col, val, xm), orc.abs_csr(row, col, val, xm),
                          TOL_F64 if val_kind == "f64" else TOL_F32, what=f"matrix {m} rep {rep}")
    # plain launch gives the same bits
    y2 = p.spmv(xt)
    assert np.array_equal(y2.cpu().numpy(), yh)


def test_blockdiag_structure(batch_env):
    torch, D, F, orc, mats, big, off, x = batch_env
    assert big.n == sum(len(r) - 1 for r, _, _ in mats) and big.nnz == sum(len(c) for _, c, _ in mats)
    for m, (row, col, val) in enumerate(mats):
        a = int(off[m])
        r0 = int(big.row[a])
        np.testing.assert_array_equal(big.col[r0:r0 + len(col)], col.astype(np.int64) + a)


def test_autotune_picks_and_caches(tmp_path, monkeypatch):
    """The tuner times every candidate, picks the fastest, caches it per
    signature, and the tuned plan is at parity."""
    import torch

    from int_spmv_b200 import autotune as T
    from int_spmv_b200 import formats as F
    from int_spmv_b200 import matrices as M
    from oracle import Oracle
    monkeypatch.setenv("ISPMV_TUNE_CACHE", str(tmp_path / "tune.json"))
    row, col, val = M.random_csr(20000, 5, rl_max=40, empty_frac=0.02)
    csr = F.CSR(row, col, val)
    x = M.uniform_x(20000, 5)
    c1 = T.tune(csr, x, reps=5)
    assert not c1["cached"] and len(c1["timings"]) >= 8
    assert c1["seconds"] == min(t["seconds"] for t in c1["timings"])
    c2 = T.tune(csr, x, reps=5)
    assert c2["cached"] and c2["format"] == c1["format"] and c2["kwargs"] == c1["kwargs"]
    p, _ = T.best_plan(csr, x)
    orc = Oracle()
    y = p.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
    assert_parity(y, orc.cf_csr(row, col, val, x), orc.abs_csr(row, col, val, x), TOL_F64, what="tuned plan")
    ck = T.tune(csr, x, k=16, reps=3)
    assert ck["kwargs"]["rhs_block"] in (8, 16, 32)


@pytest.mark.parametrize("val_kind,kw", [("f32", dict(kernel="wide")), ("f32", dict(kernel="wide", variant=32)),
                                         ("f64", dict(kernel="wide", variant=26)), ("f64", dict(kernel="ldg", variant=16)),
                                         ("f32", dict(kernel="ldg", variant=16))])
def test_graph_capture_as_first_product(val_kind, kw):
    """A plan whose first product is the graph launch: its per-product work
    areas (the FP32 copy of x) exist before the capture begins, and the
    captured graph gives the oracle's product; plain products after it too."""
    import torch

    from int_spmv_b200 import device as D
    from int_spmv_b200 import formats as F
    from int_spmv_b200 import matrices as M
    from oracle import Oracle
    row, col, val = M.random_csr(30011, 9, rl_max=40, empty_frac=0.05)
    x = M.uniform_x(30011, 9)
    csr = F.CSR(row, col, val)
    orc = Oracle()
    ref, ab = orc.cf_csr(row, col, val, x), orc.abs_csr(row, col, val, x)
    tol = TOL_F64 if val_kind == "f64" else TOL_F32
    p = D.Plan(csr, F.getFormatDataAXT(0, 128, 8, 1, "COM", csr, x)[1], val=val_kind, **kw)
    xt = torch.from_numpy(x).cuda()
    y = torch.full((30011,), 3.0, dtype=torch.float64, device="cuda")
    p.spmv_graph(xt, y)
    assert_parity(y.cpu().numpy(), ref, ab, tol, what=f"graph first {val_kind} {kw}")
    assert_parity(p.spmv(xt).cpu().numpy(), ref, ab, tol, what=f"plain after graph {val_kind} {kw}")
