"""Parity helpers shared by the GPU tests.

The bound is componentwise: |y_i - y_ref_i| <= tol * (|A| |x|)_i, with
tol = 1e-12 for FP64 values and 1e-6 for the FP32-value forms (their
products are rounded to FP32; accumulation stays FP64).  y_ref is the
oracle's naive CSR product (oracle.c, bit-exact to the reference's
cf_CSR, intSpmv_main.c:382-396)."""
from __future__ import annotations

import numpy as np

TOL_F64 = 1e-12
TOL_F32 = 1e-6


def parity_report(y, y_ref, absax, tol):
    y, y_ref, absax = (np.asarray(a, np.float64) for a in (y, y_ref, absax))
    err = np.abs(y - y_ref)
    bound = tol * absax
    bad = err > bound
    worst = int(np.argmax(err - bound)) if len(err) else 0
    return bool(bad.any()), dict(nbad=int(bad.sum()), worst=worst, err=float(err[worst]) if len(err) else 0.0,
                                 bound=float(bound[worst]) if len(err) else 0.0)


def assert_parity(y, y_ref, absax, tol=TOL_F64, what=""):
    bad, rep = parity_report(y, y_ref, absax, tol)
    assert not bad, f"{what}: {rep}"
