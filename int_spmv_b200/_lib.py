"""Loads libintspmv.so (built in-tree by int_spmv_b200.build) and binds the
C ABI of include/intspmv.h.  There is no fallback: a missing or stale
library is an error."""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

from . import abi

LIB_PATH = Path(__file__).resolve().parent / "libintspmv.so"
_lock = threading.Lock()
_lib: C.CDLL | None = None


class IntSpmvError(RuntimeError):
    """A non-zero status from the C ABI (ISPMV_ERR_*)."""

    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        msg = f"{where}: {status_string(status)}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise ImportError(f"{LIB_PATH} is missing: build it with `python -m int_spmv_b200.build` "
                                  "(requires nvcc); there is no CPU fallback")
            lib = C.CDLL(str(LIB_PATH))
            for name, (res, args) in abi.PROTOTYPES.items():
                fn = getattr(lib, name)  # AttributeError = stale library
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def status_string(st: int) -> str:
    return load().ispmv_status_string(st).decode()


def last_error() -> str:
    return load().ispmv_last_error().decode()


def check(st: int, where: str) -> None:
    if st != abi.OK:
        raise IntSpmvError(st, where, last_error() if st == abi.ERR_CUDA else "")


def launch_count() -> int:
    return int(load().ispmv_launch_count())
