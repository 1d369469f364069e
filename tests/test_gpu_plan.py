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

# (format, kernel) pairs a plan supports: "rows" = the row-parallel kernels,
# "ldg" / "tma" = the slot-stream (or tile-column) kernels with plain loads /
# 1D bulk copies.
COMBOS = [("CSR", "rows"), ("CSR", "ldg"), ("CSR", "tma"), ("AXC", "rows"), ("AXC", "ldg"), ("AXC", "tma"),
          ("K1", "auto"), ("K1P", "auto"), ("NOC1", "ldg"), ("NOC1", "tma"), ("NOC4", "ldg"), ("NOC4", "tma"),
          ("NOC8", "ldg"), ("NOC8", "tma"), ("NOC16", "ldg"), ("NOC16", "tma"), ("NOC3", "ldg"),
          ("COM128", "ldg"), ("COM128", "tma"), ("COM256", "ldg"), ("COM512", "tma"),
          ("COM128", "wide"), ("NOC1", "wide"), ("AXC", "wide"), ("CSR", "wide"), ("NOC4", "wide"), ("NOC8", "wide"),
          ("NOC3", "wide"), ("NOC16", "auto"), ("CSR", "auto"), ("AXC", "auto")]
KIDS = {"ldg": 1, "tma": 2, "rows": 3, "wide": 4}
# the lane-interleaved kernel variants the library runs (0, 8, 9: 16 slots per
# lane at three segment sizes; 4: 8 slots; 11: bulk-copy staged; 16: texture
# gathers; 18-21: TMEM-staged; 26: per-CTA x window; 32: column prefetch)
WIDE_VARIANTS = [0, 4, 8, 9, 11, 16, 18, 19, 20, 21, 26, 32]


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


def check_plan(env, row, colidx, val, x, fmt, val_kind="f64", beta=0, **kw):
    torch, D, F, orc = env
    csr = F.CSR(row, colidx, val)
    p = make_plan(F, D, csr, x, fmt, val=val_kind, **kw)
    n = csr.n
    xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    y0 = np.random.default_rng(5).uniform(-1, 1, n)
    yt = torch.from_numpy(y0.copy()).cuda()
    p.spmv(xt, yt, beta=beta)
    y = yt.cpu().numpy()
    ref = orc.cf_csr(row, colidx, val, x) + (y0 if beta else 0.0)
    absax = orc.abs_csr(row, colidx, val, x) + (np.abs(y0) * 1e-4 if beta else 0.0)
    assert_parity(y, ref, absax, TOL_F64 if val_kind == "f64" else TOL_F32, what=f"{fmt}/{val_kind}/beta{beta}")
    return p, xt


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("fmt,kernel", COMBOS)
@pytest.mark.parametrize("val_kind", ["f64", "f32"])
def test_golden(env, name, fmt, kernel, val_kind):
    g = load_golden(name)
    for beta in (0, 1):
        p, _ = check_plan(env, g["row"], g["col"], g["val"], g["x"], fmt, val_kind, beta, kernel=kernel)
        if kernel in KIDS:
            assert p.info["kernel"] == KIDS[kernel]
    assert p.status() == 0


@pytest.mark.parametrize("fmt,kernel", COMBOS)
def test_segment_boundaries(env, fmt, kernel):
    """Small warp segments and long rows: rows span many segments."""
    from int_spmv_b200 import matrices as M
    row, col, val = M.random_csr(3001, 9, rl_max=700, empty_frac=0.2)
    x = M.uniform_x(3001, 9)
    for upw in (32, 64, 0):
        check_plan(env, row, col, val, x, fmt, units_per_warp=upw, kernel=kernel)


@pytest.mark.parametrize("fmt", ["COM128", "NOC1", "AXC", "CSR"])
@pytest.mark.parametrize("variant", [0, 2, 12])
def test_stream_variants(env, fmt, variant):
    """The first slot-stream kernel: 4 slots per lane at 5 or 6 CTAs per SM,
    with L2 prefetch of the stream (12); the bulk-copy staged form."""
    from int_spmv_b200 import matrices as M
    row, col, val = M.random_csr(7001, 12, rl_max=90, empty_frac=0.1)
    x = M.uniform_x(7001, 12)
    check_plan(env, row, col, val, x, fmt, kernel="ldg", variant=variant)
    if variant == 0:
        for ctas in (0, 1):
            p, _ = check_plan(env, row, col, val, x, fmt, kernel="tma", variant=variant, ctas_per_sm=ctas)
            assert p.status() == 0


@pytest.mark.parametrize("fmt", ["COM128", "NOC1", "AXC", "CSR"])
@pytest.mark.parametrize("variant", WIDE_VARIANTS)
@pytest.mark.parametrize("val_kind", ["f64", "f32"])
def test_wide_variants(env, fmt, variant, val_kind):
    """Every lane-interleaved kernel variant (8 or 16 slots per lane, plain,
    staged, texture, TMEM, x window, column prefetch) on random rows, long
    rows spanning segments, a banded matrix with empty rows and a 27-point
    stencil."""
    from int_spmv_b200 import matrices as M
    mats = [M.random_csr(7001, 12, rl_max=90, empty_frac=0.1), M.random_csr(3001, 9, rl_max=700, empty_frac=0.2),
            M.fem_banded(20011, np.random.default_rng(5), 3, 30), M.stencil27(22, seed=2)]
    for i, (row, col, val) in enumerate(mats):
        x = M.uniform_x(len(row) - 1, 12 + i)
        for beta in (0, 1):
            p, _ = check_plan(env, row, col, val, x, fmt, val_kind, beta, kernel="wide", variant=variant)
            assert p.info["kernel"] == 4 and p.kernel_name().startswith(("stream_wide", "stream_tmem"))


def test_wide_rejects_other_forms(env):
    torch, D, F, orc = env
    from int_spmv_b200 import IntSpmvError
    g = load_golden("random257_empty")
    csr = F.CSR(g["row"], g["col"], g["val"])
    with pytest.raises(IntSpmvError):
        make_plan(F, D, csr, g["x"], "COM128", col="d16", kernel="wide", variant=26)  # x window: u32 columns only
    with pytest.raises(IntSpmvError):
        make_plan(F, D, csr, g["x"], "COM128", col="d16", kernel="wide", variant=11)  # bulk-copy stages: u32 only
    with pytest.raises(IntSpmvError):
        make_plan(F, D, csr, g["x"], "COM128", val="f32lo", kernel="wide", variant=32)  # column prefetch: no lo-words
    with pytest.raises(IntSpmvError):
        make_plan(F, D, csr, g["x"], "COM128", val="f32lo", kernel="wide", variant=16)  # texture gathers: no lo-words
    for v in (1, 2, 22, 34, 99):  # not a variant this library runs
        with pytest.raises(IntSpmvError):
            make_plan(F, D, csr, g["x"], "COM128", kernel="wide", variant=v)


WIDE_D16 = [0, 4, 8, 9, 16]


@pytest.mark.parametrize("fmt", ["COM128", "NOC1", "CSR"])
@pytest.mark.parametrize("variant", WIDE_D16)
@pytest.mark.parametrize("val_kind", ["f64", "f32"])
def test_wide_d16(env, fmt, variant, val_kind):
    """16-bit column deltas per batch of the lane-interleaved kernel: banded
    matrices (deltas), random ones (batches escape to u32 columns) and long
    rows spanning segments."""
    from int_spmv_b200 import matrices as M
    mats = [M.fem_banded(20011, np.random.default_rng(5), 3, 30), M.stencil27(22, seed=2),
            M.random_csr(7001, 12, rl_max=90, empty_frac=0.1), M.random_csr(3001, 9, rl_max=700, empty_frac=0.2)]
    for i, (row, col, val) in enumerate(mats):
        x = M.uniform_x(len(row) - 1, 30 + i)
        for beta in (0, 1):
            p, _ = check_plan(env, row, col, val, x, fmt, val_kind, beta, kernel="wide", variant=variant, col="d16")
            assert p.info["kernel"] == 4 and p.info["col_kind"] == 1 and "d16" in p.kernel_name()


WIDE_LO = [0, 4, 8, 9]


@pytest.mark.parametrize("fmt", ["COM128", "NOC1", "CSR"])
@pytest.mark.parametrize("variant", WIDE_LO)
@pytest.mark.parametrize("col_kind", ["u32", "d16"])
def test_wide_lo(env, fmt, variant, col_kind):
    """BF16 lo-words on the lane-interleaved kernel (FP32 values, FP64 x):
    the default tolerance (flagged segments only) and every row flagged
    (hi + lo within 1e-8), on banded, stencil, random and long-row matrices."""
    torch, D, F, orc = env
    from int_spmv_b200 import matrices as M
    mats = [M.fem_banded(20011, np.random.default_rng(5), 3, 30), M.stencil27(22, seed=2),
            M.random_csr(7001, 12, rl_max=90, empty_frac=0.1), M.random_csr(3001, 9, rl_max=700, empty_frac=0.2)]
    for i, (row, col, val) in enumerate(mats):
        x = M.uniform_x(len(row) - 1, 40 + i)
        for beta in (0, 1):
            p, _ = check_plan(env, row, col, val, x, fmt, "f32lo", beta, kernel="wide", variant=variant, col=col_kind)
            assert p.info["kernel"] == 4 and p.kernel_name().endswith("lo>")
        csr = F.CSR(row, col, val)
        p = make_plan(F, D, csr, x, fmt, val="f32lo", kernel="wide", variant=variant, col=col_kind, lo_tol=1e-300)
        y = p.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
        assert_parity(y, orc.cf_csr(row, col, val, x), orc.abs_csr(row, col, val, x), 1e-8,
                      what=f"{fmt} wide v{variant} f32lo all rows")


@pytest.mark.parametrize("fmt", ["COM128", "NOC1"])
def test_auto_picks_wide(env, fmt):
    """AXT COM and tileH=1 plans default to the lane-interleaved kernel: 16
    slots per lane for rows of 16+ nonzeros (bulk-copy staged unless the
    columns are scattered), 8 for short rows (where the columns are uniformly
    scattered, not on fixed far diagonals: per-CTA x windows for FP64 values,
    column prefetch for FP32 values), u32 or 16-bit columns, and the BF16
    lo-word form."""
    torch, D, F, orc = env
    from int_spmv_b200 import matrices as M
    for rl_max, name in ((8, "stream_wide<8,stg"), (60, "stream_wide<16,")):
        row, col, val = M.random_csr(5000, rl_max, rl_max=rl_max, empty_frac=0.05)
        x = M.uniform_x(5000, rl_max)
        p, _ = check_plan(env, row, col, val, x, fmt)
        assert p.info["kernel"] == 4 and p.kernel_name().startswith(name), p.kernel_name()
        if rl_max == 8:  # FP32 values, scattered short rows: the next batch's columns loaded ahead
            p, _ = check_plan(env, row, col, val, x, fmt, val_kind="f32")
            assert p.kernel_name().startswith("stream_wide<8,w0,b4,pfc>"), p.kernel_name()
        if rl_max > 8:
            p, _ = check_plan(env, row, col, val, x, fmt, val_kind="f32")
            assert p.kernel_name().startswith("stream_wide<16,")
        p, _ = check_plan(env, row, col, val, x, fmt, col="d16")
        assert p.info["kernel"] == 4 and p.kernel_name().endswith("d16>")
        p, _ = check_plan(env, row, col, val, x, fmt, val_kind="f32lo")
        assert p.info["kernel"] == 4 and p.kernel_name().endswith("lo>")
    # short rows whose far columns sit on fixed diagonals (+-1700): neighbouring
    # rows share lines, so no per-CTA window
    n = 20000
    r = np.repeat(np.arange(n), 3)
    c = (r + np.tile([-1700, 0, 1700], n)) % n
    order = np.lexsort((c, r))
    row = np.arange(0, 3 * n + 1, 3, dtype=np.uint32)
    col, val = c[order].astype(np.uint32), np.random.default_rng(2).normal(size=3 * n)
    p, _ = check_plan(env, row, col, val, M.uniform_x(n, 2), fmt)
    assert p.kernel_name().startswith("stream_wide<8,w0"), p.kernel_name()
    # long rows whose columns are not scattered (27-point stencil): the
    # bulk-copy staged stream
    row, col, val = M.stencil27(20, seed=2)
    p, _ = check_plan(env, row, col, val, M.uniform_x(8000, 2), fmt)
    assert p.kernel_name().startswith("stream_wide_tma<16,"), p.kernel_name()


@pytest.mark.parametrize("fmt,kernel", [("NOC1", "ldg"), ("NOC4", "tma"), ("COM128", "ldg"), ("COM128", "tma"),
                                        ("CSR", "rows"), ("K1P", "auto"), ("COM128", "wide"), ("CSR", "wide")])
def test_deterministic_and_host_e2e(env, fmt, kernel):
    torch, D, F, orc = env
    from int_spmv_b200 import matrices as M
    row, col, val = M.random_csr(20000, 4, rl_max=60, empty_frac=0.05)
    x = M.uniform_x(20000, 4)
    p, xt = check_plan(env, row, col, val, x, fmt, kernel=kernel)
    a = p.spmv(xt).cpu().numpy()
    b = p.spmv(xt).cpu().numpy()
    assert np.array_equal(a, b)  # no atomics on the plan path: bitwise repeatable
    hx = torch.from_numpy(x.copy()).pin_memory()
    hy = torch.empty(20000, dtype=torch.float64).pin_memory()
    p.spmv_host(hx, hy)
    assert np.array_equal(hy.numpy(), a)


@pytest.mark.parametrize("fmt,kernel,val_kind", [("COM128", "auto", "f64"), ("COM128", "auto", "f32"),
                                                 ("K1", "auto", "f64"), ("NOC4", "ldg", "f64")])
def test_time_main(env, fmt, kernel, val_kind):
    """ispmv_plan_time_main: a positive mean time for the main kernel alone;
    it rejects a bad repetition count, and a product after it is the oracle's
    (the timing leaves the fix-up rows out of y, spmv puts them back)."""
    torch, D, F, orc = env
    from int_spmv_b200 import matrices as M
    from int_spmv_b200._lib import IntSpmvError
    row, col, val = M.random_csr(30000, 6, rl_max=90, empty_frac=0.05)
    x = M.uniform_x(30000, 6)
    p, xt = check_plan(env, row, col, val, x, fmt, val_kind=val_kind, kernel=kernel)
    y = torch.empty(30000, dtype=torch.float64, device="cuda")
    ms = p.time_main(xt, y, 5)
    assert 0.0 < ms < 1e3
    with pytest.raises(IntSpmvError):
        p.time_main(xt, y, 0)
    p.spmv(xt, y)
    assert_parity(y.cpu().numpy(), orc.cf_csr(row, col, val, x), orc.abs_csr(row, col, val, x),
                  TOL_F64 if val_kind == "f64" else TOL_F32, what=f"after time_main {fmt}/{val_kind}")


@pytest.fixture(scope="module")
def poisson512(env):
    from int_spmv_b200 import matrices as M
    row, col, val = M.poisson2d(512)
    return row, col, val, M.uniform_x(len(row) - 1, 0)


@pytest.mark.parametrize("fmt,kernel", [("CSR", "rows"), ("NOC1", "ldg"), ("NOC1", "tma"), ("COM128", "ldg"),
                                        ("NOC1", "wide"), ("COM128", "wide")])
def test_poisson512(env, poisson512, fmt, kernel):
    row, col, val, x = poisson512
    assert len(row) - 1 == 262144 and len(col) == 1308672
    check_plan(env, row, col, val, x, fmt, kernel=kernel)


@pytest.fixture(scope="module")
def powerlaw4m(env):
    from int_spmv_b200 import matrices as M
    row, col, val = M.powerlaw(4_000_000, seed=1)
    return row, col, val, M.uniform_x(4_000_000, 1)


@pytest.mark.parametrize("fmt,kernel", [("CSR", "rows"), ("CSR", "ldg"), ("AXC", "rows"), ("AXC", "ldg"),
                                        ("K1P", "auto"), ("NOC1", "ldg"), ("NOC1", "tma"), ("NOC4", "ldg"),
                                        ("NOC4", "tma"), ("NOC8", "tma"), ("COM128", "ldg"), ("COM128", "tma"),
                                        ("COM512", "ldg"), ("COM128", "wide"), ("NOC1", "wide"), ("CSR", "wide"),
                                        ("NOC4", "auto"), ("NOC8", "auto"), ("AXC", "auto"), ("K1", "auto")])
def test_powerlaw_4m(env, powerlaw4m, fmt, kernel):
    row, col, val, x = powerlaw4m
    p, _ = check_plan(env, row, col, val, x, fmt, kernel=kernel)
    assert p.status() == 0
    if (fmt, kernel) in (("COM128", "ldg"), ("NOC1", "ldg"), ("COM128", "wide"), ("NOC4", "auto"), ("K1", "auto")):
        check_plan(env, row, col, val, x, fmt, val_kind="f32", kernel=kernel)


STREAM_FMTS = [("COM128", "ldg"), ("NOC1", "ldg"), ("AXC", "ldg"), ("CSR", "ldg")]
NARROW = [("f32lo", "u32"), ("f32", "d16"), ("f64", "d16"), ("f32lo", "d16")]


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("fmt,kernel", STREAM_FMTS)
@pytest.mark.parametrize("val_kind,col_kind", NARROW)
def test_precision_forms_golden(env, name, fmt, kernel, val_kind, col_kind):
    g = load_golden(name)
    for beta in (0, 1):
        check_plan(env, g["row"], g["col"], g["val"], g["x"], fmt, val_kind, beta, kernel=kernel, col=col_kind)


@pytest.mark.parametrize("fmt,kernel", STREAM_FMTS)
def test_precision_forms_banded_and_random(env, fmt, kernel):
    """Banded rows (16-bit deltas fit) and random rows (batches escape to u32);
    with every row carrying a lo-word the FP32 + BF16 form is within 1e-8."""
    torch, D, F, orc = env
    from int_spmv_b200 import matrices as M
    rng = np.random.default_rng(3)
    mats = [M.fem_banded(5000, rng), M.random_csr(6000, 21, rl_max=50, empty_frac=0.05), M.stencil27(20, seed=2)]
    for row, col, val in mats:
        x = M.uniform_x(len(row) - 1, 8)
        for vk, ck in NARROW:
            p, _ = check_plan(env, row, col, val, x, fmt, vk, kernel=kernel, col=ck)
            assert p.info["col_kind"] == (1 if ck == "d16" else 0)
        # all rows flagged: residual-corrected values
        csr = F.CSR(row, col, val)
        p = make_plan(F, D, csr, x, fmt, val="f32lo", kernel=kernel, lo_tol=1e-300)
        y = p.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
        assert_parity(y, orc.cf_csr(row, col, val, x), orc.abs_csr(row, col, val, x), 1e-8, what=f"{fmt} f32lo all")


def test_precision_forms_rejected_elsewhere(env):
    torch, D, F, orc = env
    from int_spmv_b200 import IntSpmvError
    g = load_golden("random257_empty")
    csr = F.CSR(g["row"], g["col"], g["val"])
    with pytest.raises(IntSpmvError):
        make_plan(F, D, csr, g["x"], "K1P", col="d16")
    with pytest.raises(IntSpmvError):
        make_plan(F, D, csr, g["x"], "NOC4", val="f32lo", kernel="ldg")
    with pytest.raises(IntSpmvError):
        make_plan(F, D, csr, g["x"], "CSR", col="d16", kernel="rows")


@pytest.mark.parametrize("fmt,kernel", [("COM128", "ldg"), ("NOC4", "tma"), ("K1", "auto"), ("CSR", "rows")])
def test_kernel_timing_events(env, fmt, kernel):
    """Event pairs around the main kernel: one pair per spmv (a ring of the
    latest), none for graph launches, and the product unchanged."""
    torch, D, F, orc = env
    from int_spmv_b200 import matrices as M
    row, col, val = M.random_csr(50000, 21, rl_max=40)
    x = M.uniform_x(50000, 21)
    csr = F.CSR(row, col, val)
    p = make_plan(F, D, csr, x, fmt, kernel=kernel)
    xt = torch.from_numpy(x).cuda()
    y = torch.empty_like(xt)
    p.time_kernels(4)
    for _ in range(6):
        p.spmv(xt, y)
    torch.cuda.synchronize()
    ms, n = p.kernel_ms()
    assert n == 4 and ms > 0
    assert p.kernel_name()
    p.spmv_graph(xt, y)
    torch.cuda.synchronize()
    assert p.kernel_ms() == (0.0, 0)
    p.time_kernels(0)
    p.spmv(xt, y)
    torch.cuda.synchronize()
    assert p.kernel_ms() == (0.0, 0)
    assert_parity(y.cpu().numpy(), orc.cf_csr(row, col, val, x), orc.abs_csr(row, col, val, x), TOL_F64)


@pytest.mark.parametrize("val_kind", ["f64", "f32"])
def test_wide_texture_gathers_and_fallback(env, val_kind):
    """Texture-gather variants: an aligned x is fetched through a linear
    texture; an x that does not meet the texture alignment (a view 8 bytes
    into a buffer) is gathered with loads; both give the oracle's product."""
    torch, D, F, orc = env
    from int_spmv_b200 import matrices as M
    row, col, val = M.random_csr(5003, 3, rl_max=40, empty_frac=0.05)
    x = M.uniform_x(5003, 3)
    csr = F.CSR(row, col, val)
    ref, ab = orc.cf_csr(row, col, val, x), orc.abs_csr(row, col, val, x)
    tol = TOL_F64 if val_kind == "f64" else TOL_F32
    for variant in (16,):
        p = make_plan(F, D, csr, x, "COM128", kernel="wide", variant=variant, val=val_kind)
        y = p.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
        if val_kind == "f64":
            assert p.kernel_name().endswith("tex>"), p.kernel_name()
        assert_parity(y, ref, ab, tol, what=f"tex v{variant}")
        buf = torch.zeros(5004, dtype=torch.float64, device="cuda")
        buf[1:] = torch.from_numpy(x).cuda()
        y2 = p.spmv(buf[1:]).cpu().numpy()
        if val_kind == "f64":
            assert "gathered with loads" in p.kernel_name(), p.kernel_name()
        assert_parity(y2, ref, ab, tol, what=f"tex fallback v{variant}")
        # a captured graph gathers with loads (it must not name a texture a
        # later product replaces), and later products with other x stay right
        xa = torch.from_numpy(x).cuda()
        yg = torch.empty_like(xa)
        p.spmv_graph(xa, yg)
        p.spmv(buf[1:])
        p.spmv_graph(xa, yg)
        assert_parity(yg.cpu().numpy(), ref, ab, tol, what=f"tex graph v{variant}")


@pytest.mark.gpu
@pytest.mark.parametrize("val_kind", ["f64", "f32"])
@pytest.mark.parametrize("variant", [26])
def test_wide_staged_window(env, val_kind, variant):
    """Per-CTA x windows copied by one bulk copy: a banded matrix (most
    columns inside a CTA's window) and a matrix of uniform columns (most
    outside), n odd (the last x element is never in a window), with an
    aligned x (the staged kernel) and an x 8 bytes into a buffer (no bulk
    copy: plain loads over the same stream)."""
    torch, D, F, orc = env
    from int_spmv_b200 import matrices as M
    mats = [M.powerlaw(30001, seed=7, band=300), M.random_csr(20011, 4, rl_max=60, empty_frac=0.05)]
    tol = TOL_F64 if val_kind == "f64" else TOL_F32
    for row, col, val in mats:
        n = len(row) - 1
        x = M.uniform_x(n, 5)
        csr = F.CSR(row, col, val)
        ref, ab = orc.cf_csr(row, col, val, x), orc.abs_csr(row, col, val, x)
        p = make_plan(F, D, csr, x, "COM128", kernel="wide", variant=variant, val=val_kind)
        y = p.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
        assert "stg" in p.kernel_name(), p.kernel_name()
        assert_parity(y, ref, ab, tol, what=f"staged v{variant}")
        buf = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
        buf[1:] = torch.from_numpy(x).cuda()
        y2 = p.spmv(buf[1:]).cpu().numpy()
        assert "stg" not in p.kernel_name(), p.kernel_name()
        assert_parity(y2, ref, ab, tol, what=f"staged fallback v{variant}")
        yt = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, n)).cuda()
        y0 = yt.cpu().numpy()
        p.spmv(torch.from_numpy(x).cuda(), yt, beta=1)
        assert_parity(yt.cpu().numpy(), ref + y0, ab + np.abs(y0) * 1e-4, tol, what=f"staged beta1 v{variant}")
        assert p.status() == 0
