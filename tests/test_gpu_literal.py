"""sm_100a kernels on the reference's own arrays (x-baked ax, sec
descriptors, K1 chunks) against the oracle's CSR product, on every golden
fixture; and the reference-named host-pointer entry points."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import golden_names, load_golden
from paritylib import assert_parity

pytestmark = pytest.mark.gpu

AXT_CASES = [("NOC", 1, 128), ("NOC", 4, 128), ("NOC", 8, 128), ("NOC", 16, 128), ("NOC", 48, 128), ("NOC", 3, 128),
             ("COM", 1, 128), ("COM", 1, 256), ("COM", 1, 512), ("COM", 1, 8)]


@pytest.fixture(scope="module")
def env():
    import torch
    from int_spmv_b200 import device as D
    from oracle import Oracle
    return torch, D, Oracle()


def _abs(orc, g):
    return orc.abs_csr(g["row"], g["col"], g["val"], g["x"])


@pytest.mark.parametrize("name", golden_names())
def test_cf_csr_axc_k1(env, name):
    torch, D, orc = env
    g = load_golden(name)
    n = len(g["rl"])
    absax = _abs(orc, g)
    T = D.to_device
    y = torch.full((n,), 7.0, dtype=torch.float64, device="cuda")
    D.cf_CSR(T(g["row"]), T(g["col"]), T(g["val"]), T(g["x"]), y)
    assert_parity(y.cpu().numpy(), g["y_csr"], absax, what="cf_CSR")
    y.fill_(7.0)
    D.int_axc(n, T(g["axc_ax"]), T(g["axc_brp"]), y)
    assert_parity(y.cpu().numpy(), g["y_csr"], absax, what="int_axc")
    cn = len(g["k1_nmc"])
    res = torch.zeros(cn * 8, dtype=torch.float64, device="cuda")
    args = (T(g["k1_val"]), T(g["k1_col"]), T(g["k1_chp"]), T(g["k1_nmc"]))
    D.int_k1(cn, *args, T(g["x"]), res)
    assert np.allclose(res.cpu().numpy(), g["k1_res"], rtol=0, atol=1e-12 * max(1.0, absax.max()))
    y.fill_(7.0)
    D.orderArrayK1(n, T(g["k1_permi"]), res, y)
    assert_parity(y.cpu().numpy(), g["y_csr"], absax, what="int_k1+orderArrayK1")
    y.fill_(7.0)
    D.int_k1p(int(g["k1_mask"]), cn, *args, T(g["k1_permi"]), T(g["x"]), y)
    assert_parity(y.cpu().numpy(), g["y_csr"], absax, what="int_k1p")


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("mode,th,bs", AXT_CASES)
def test_axt(env, name, mode, th, bs):
    torch, D, orc = env
    g = load_golden(name)
    n = len(g["rl"])
    key = f"axt_{mode}_{th}_{bs}"
    tileN, lenAX, lenSEC, _, log, _ = (int(v) for v in g[key + "_meta"])
    ax, sec = D.to_device(g[key + "_ax"]), D.to_device(g[key + "_sec"])
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    if mode == "COM":
        bn = (tileN * 8 + bs - 1) // bs
        D.int_axt_com_h1(bn, bs, log, 8, tileN, lenAX, lenSEC, ax, sec, y)
    elif th == 1:
        D.int_axt_noc_h1(tileN, ax, sec, y)
    else:
        D.int_axt_noc(tileN, th, ax, sec, y)
    # the compacted kernel is judged against the CSR oracle (the reference's
    # own result drops row-0 segments, README.md:33)
    assert_parity(y.cpu().numpy(), g["y_csr"], _abs(orc, g), what=key)


@pytest.mark.parametrize("name", ["random257_empty", "row0_129", "one_by_one"])
def test_reference_names_on_host_pointers(env, name):
    """cf_CSR, int_axc, int_k1/orderArrayK1, int_k1p and the AXT kernels by
    their reference names and signatures, on host arrays."""
    torch, D, orc = env
    from int_spmv_b200 import abi
    from int_spmv_b200._lib import load
    lib = load()
    g = load_golden(name)
    n = len(g["rl"])
    absax = _abs(orc, g)
    P_D, P_U = abi.P_FPT, abi.P_UIN

    def pd(a):
        return np.ascontiguousarray(a, np.float64).ctypes.data_as(P_D)

    def pu(a):
        return np.ascontiguousarray(a, np.uint32).ctypes.data_as(P_U)

    row, col, val, x = g["row"], g["col"], g["val"], g["x"]
    s = abi.StrMatCSR()
    s.nrows, s.nnz = n, len(col)
    s.row, s.col, s.val = pu(row), pu(col), pd(val)
    y = np.zeros(n)
    lib.cf_CSR(s, pd(x), y.ctypes.data_as(P_D))
    assert_parity(y, g["y_csr"], absax, what="cf_CSR(host)")
    y = np.zeros(n)
    lib.int_axc(1, n, pd(g["axc_ax"]), pu(g["axc_brp"]), y.ctypes.data_as(P_D))
    assert_parity(y, g["y_csr"], absax, what="int_axc(host)")
    cn = len(g["k1_nmc"])
    res = np.zeros(cn * 8)
    kv, kc, kchp, knmc = (np.ascontiguousarray(g[k]) for k in ("k1_val", "k1_col", "k1_chp", "k1_nmc"))
    lib.int_k1(1, cn, pd(kv), pu(kc), pu(kchp), pu(knmc), pd(x), res.ctypes.data_as(P_D))
    y = np.zeros(n)
    lib.orderArrayK1(1, n, pu(g["k1_permi"]), res.ctypes.data_as(P_D), y.ctypes.data_as(P_D))
    assert_parity(y, g["y_csr"], absax, what="int_k1(host)")
    y = np.zeros(n + 1)
    lib.int_k1p(1, int(g["k1_mask"]), cn, pd(kv), pu(kc), pu(kchp), pu(knmc), pu(g["k1_permi"]), pd(x),
                y.ctypes.data_as(P_D))
    assert_parity(y[:n], g["y_csr"], absax, what="int_k1p(host)")
    for mode, th, bs in [("NOC", 1, 128), ("NOC", 8, 128), ("COM", 1, 256)]:
        key = f"axt_{mode}_{th}_{bs}"
        tileN, lenAX, lenSEC, _, log, _ = (int(v) for v in g[key + "_meta"])
        y = np.zeros(n)
        ax, sec = np.ascontiguousarray(g[key + "_ax"]), np.ascontiguousarray(g[key + "_sec"])
        if mode == "COM":
            lib.int_axt_com_h1(1, (tileN * 8 + bs - 1) // bs, bs, log, 8, tileN, lenAX, lenSEC, pd(ax), pu(sec),
                               y.ctypes.data_as(P_D))
        elif th == 1:
            lib.int_axt_noc_h1(1, tileN, pd(ax), pu(sec), y.ctypes.data_as(P_D))
        else:
            lib.int_axt_noc(1, tileN, th, pd(ax), pu(sec), y.ctypes.data_as(P_D))
        assert_parity(y, g["y_csr"], absax, what=key + "(host)")


def test_literal_rejects_bad_arguments(env):
    torch, D, orc = env
    from int_spmv_b200 import IntSpmvError
    ax = torch.zeros(16, dtype=torch.float64, device="cuda")
    sec = torch.zeros(8, dtype=torch.int32, device="cuda")
    y = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(IntSpmvError):
        D.int_axt_com_h1(1, 100, 7, 8, 1, 16, 8, ax, sec, y)  # bs not a power of two
    with pytest.raises(IntSpmvError):
        D.int_axt_com_h1(1, 128, 7, 4, 1, 16, 8, ax, sec, y)  # tile width other than 8
    with pytest.raises(IntSpmvError):
        D.int_axt_com_h1(1, 1024, 10, 8, 1, 16, 8, ax, sec, y)  # bs beyond the reference's 512
