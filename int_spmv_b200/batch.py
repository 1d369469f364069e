"""Batched SpMV over many independent (uneven) square matrices.

The matrices are assembled into one block-diagonal CSR (ispmv_csr_blockdiag),
built into one format and uploaded as one plan whose slot stream holds every
matrix's rows back to back.  One SpMV of that plan multiplies every matrix by
its own slice of x: a single launch of the work-queue kernel (persistent
warps pulling equal segments, so uneven sizes balance), or a single
CUDA-graph launch of it together with its row fix-up.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from ._lib import check, load
from .formats import CSR


def blockdiag(mats) -> tuple[CSR, np.ndarray]:
    """(block-diagonal CSR, offsets): matrix m owns rows/columns
    [off[m], off[m+1])."""
    lib = load()
    parts = [m if isinstance(m, CSR) else CSR(*m) for m in mats]
    arr = (abi.StrMatCSR * len(parts))(*[p.c for p in parts])
    out = abi.StrMatCSR()
    off = np.zeros(len(parts) + 1, dtype=np.uint32)
    check(lib.ispmv_csr_blockdiag(len(parts), arr, C.byref(out), off.ctypes.data_as(abi.P_UIN)),
          "ispmv_csr_blockdiag")
    try:
        n, nnz = out.nrows, out.nnz
        row = np.ctypeslib.as_array(out.row, shape=(n + 1,)).copy()
        col = np.ctypeslib.as_array(out.col, shape=(max(nnz, 1),))[:nnz].copy()
        val = np.ctypeslib.as_array(out.val, shape=(max(nnz, 1),))[:nnz].copy()
    finally:
        lib.ispmv_csr_free(C.byref(out))
    return CSR(row, col, val), off
