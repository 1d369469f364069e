"""Failure detection without a GPU fault: the bounded mbarrier wait that the
staged kernels (bulk-copy rings) rely on gives up on a barrier nothing
completes, reports ISPMV_ERR_TIMEOUT to the host, and leaves the context
usable for the next product."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from paritylib import TOL_F64, assert_parity

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives():
    import torch

    from int_spmv_b200 import abi
    from int_spmv_b200 import device as D
    from int_spmv_b200 import formats as F
    from int_spmv_b200 import matrices as M
    from int_spmv_b200._lib import load
    from oracle import Oracle
    lib = load()
    ms = C.c_double(-1.0)
    st = lib.ispmv_selftest_bounded_wait(C.byref(ms), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == abi.ERR_TIMEOUT, lib.ispmv_status_string(st)
    assert 50.0 <= ms.value <= 5000.0, ms.value  # gave up after its limit, not at once and not never
    # the context is intact: a staged product still runs and is right
    row, col, val = M.random_csr(20000, 17, rl_max=60, empty_frac=0.05)
    x = M.uniform_x(20000, 17)
    csr = F.CSR(row, col, val)
    _, com = F.getFormatDataAXT(0, 128, 8, 1, "COM", csr, x)
    for kernel, variant in (("tma", 0), ("wide", 11)):
        p = D.Plan(csr, com, kernel=kernel, variant=variant)
        y = p.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
        assert p.status() == 0
        orc = Oracle()
        assert_parity(y, orc.cf_csr(row, col, val, x), orc.abs_csr(row, col, val, x), TOL_F64, what=kernel)
