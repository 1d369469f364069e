"""int_spmv_b200 - a B200 (sm_100a) SpMV library that is a drop-in for the C
entry points and sparse formats of edoardoCB/int_spmv (CSR, AXC, K1, AXT).

Host side: `formats` (the reference's builders and structs, bit-exact
arrays), `matrices` (seeded synthetic workloads).  Device side: `device`
(the reference's kernels by name on device arrays) and `plan` (formats
resident in HBM; y = A x for a fresh x per call).  Everything runs through
libintspmv.so (include/intspmv.h); there is no CPU fallback.
"""
from ._lib import IntSpmvError, last_error, launch_count, load  # noqa: F401

__all__ = ["IntSpmvError", "load", "last_error", "launch_count"]
