"""The allocation-free K1 product (ispmv_dev_k1_spmv_noalloc), called
through the C ABI, against the allocating pair it replaces
(ispmv_dev_int_k1 into a caller-allocated result, then ispmv_dev_order_k1).

Callers that cannot call cudaMalloc - a solver loop whose memory is fixed
before it starts, or a host that gives the library no allocator - use the
allocation-free form; its intermediate lives in a static device array that
every call shares.  This file is collected last so a failure here cannot
stop the other tests from running; it passes alone or after them.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import load_golden
from paritylib import assert_parity

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch

    from int_spmv_b200 import device as D
    from int_spmv_b200 import formats as F
    from int_spmv_b200._lib import LIB_PATH, load
    from oracle import Oracle
    load()  # prototypes bound; the raw handle below is the same library
    lib = C.CDLL(str(LIB_PATH))
    lib.ispmv_dev_k1_spmv_noalloc.restype = C.c_int
    lib.ispmv_dev_k1_spmv_noalloc.argtypes = [C.c_uint, C.c_uint] + [C.c_void_p] * 8
    for fn in ("ispmv_dev_int_k1", "ispmv_dev_order_k1"):
        getattr(lib, fn).restype = C.c_int
    lib.ispmv_dev_int_k1.argtypes = [C.c_uint] + [C.c_void_p] * 7
    lib.ispmv_dev_order_k1.argtypes = [C.c_uint] + [C.c_void_p] * 4
    return torch, D, F, Oracle(), lib


def _k1_arrays(D, F, row, col, val, x):
    csr = F.CSR(row, col, val)
    _, k1 = F.getFormatDataK1(8, csr, x)
    T = D.to_device
    return csr.n, k1.c.chunkNum, (T(k1.val), T(k1.col), T(k1.chp), T(k1.nmc), T(k1.permi))


@pytest.mark.parametrize("case", ["random257_empty", "long_rows_700", "poisson"])
def test_noalloc_matches_allocating_pair(env, case):
    torch, D, F, orc, lib = env
    from int_spmv_b200 import matrices as M
    if case == "poisson":
        row, col, val = M.poisson2d(300)
    else:
        g = load_golden(case)
        row, col, val = g["row"], g["col"], g["val"]
    n = len(row) - 1
    for call, seed in enumerate((1, 2)):  # two calls in a row, different x
        x = M.uniform_x(n, seed)
        nrows, cn, (kval, kcol, kchp, knmc, kperm) = _k1_arrays(D, F, row, col, val, x)
        xt = torch.from_numpy(x).cuda()
        stream = torch.cuda.current_stream().cuda_stream
        # the allocating pair: K1 into a caller-allocated chunk-order array, then reorder
        res = torch.empty(cn * 8, dtype=torch.float64, device="cuda")
        y_ref = torch.full((n,), 3.0, dtype=torch.float64, device="cuda")
        assert lib.ispmv_dev_int_k1(cn, kval.data_ptr(), kcol.data_ptr(), kchp.data_ptr(), knmc.data_ptr(),
                                    xt.data_ptr(), res.data_ptr(), stream) == 0
        assert lib.ispmv_dev_order_k1(nrows, kperm.data_ptr(), res.data_ptr(), y_ref.data_ptr(), stream) == 0
        # the allocation-free form
        y = torch.full((n,), -5.0, dtype=torch.float64, device="cuda")
        assert lib.ispmv_dev_k1_spmv_noalloc(nrows, cn, kval.data_ptr(), kcol.data_ptr(), kchp.data_ptr(),
                                             knmc.data_ptr(), kperm.data_ptr(), xt.data_ptr(), y.data_ptr(),
                                             stream) == 0
        torch.cuda.synchronize()
        a, b = y.cpu().numpy(), y_ref.cpu().numpy()
        absax = orc.abs_csr(row, col, val, x)
        assert_parity(a, b, absax, what=f"noalloc vs int_k1+orderArrayK1, call {call}")
        assert_parity(a, orc.cf_csr(row, col, val, x), absax, what=f"noalloc vs oracle, call {call}")


def test_noalloc_allocates_nothing(env):
    """Repeated calls after the first leave the device's free memory as it
    was: the scratch is the static array, nothing else is allocated."""
    torch, D, F, orc, lib = env
    from int_spmv_b200 import matrices as M
    row, col, val = M.poisson2d(200)
    n = len(row) - 1
    x = M.uniform_x(n, 5)
    nrows, cn, (kval, kcol, kchp, knmc, kperm) = _k1_arrays(D, F, row, col, val, x)
    xt = torch.from_numpy(x).cuda()
    y = torch.empty(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    args = (nrows, cn, kval.data_ptr(), kcol.data_ptr(), kchp.data_ptr(), knmc.data_ptr(), kperm.data_ptr(),
            xt.data_ptr(), y.data_ptr(), stream)
    assert lib.ispmv_dev_k1_spmv_noalloc(*args) == 0  # the first call may load the library's kernels
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        assert lib.ispmv_dev_k1_spmv_noalloc(*args) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert_parity(y.cpu().numpy(), orc.cf_csr(row, col, val, x), orc.abs_csr(row, col, val, x),
                  what="noalloc after repeated calls")


def test_noalloc_rejects_beyond_maximum(env):
    torch, D, F, orc, lib = env
    from int_spmv_b200._lib import load
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = dummy.data_ptr()
    n = (1 << 20) + 1  # one row past ISPMV_K1_NOALLOC_MAX_ROWS: rejected on the host, nothing launched
    st = lib.ispmv_dev_k1_spmv_noalloc(n, (n + 7) // 8, p, p, p, p, p, p, p, None)
    assert st == 1
    assert b"ISPMV_K1_NOALLOC_MAX_ROWS" in load().ispmv_last_error()
    st = lib.ispmv_dev_k1_spmv_noalloc(16, 3, p, p, p, p, p, p, p, None)  # chunkNum != ceil(16/8)
    assert st == 1
    st = lib.ispmv_dev_k1_spmv_noalloc(16, 2, None, p, p, p, p, p, p, None)  # null values
    assert st == 1
    st = lib.ispmv_dev_k1_spmv_noalloc(16, 2, p, None, p, p, p, p, p, None)  # null columns
    assert st == 1
