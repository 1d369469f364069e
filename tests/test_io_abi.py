"""Matrix files (.csr text / .bin binary, intSpmv_main.c:187-249), the .sta
report (intSpmv_main.c:253-302), and the C ABI itself: the library loads,
exports every function include/intspmv.h declares, and its structs have the
reference's sizes."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, golden_names, load_golden
from int_spmv_b200 import IntSpmvError, abi
from int_spmv_b200 import formats as F
from int_spmv_b200._lib import LIB_PATH, load


def declared_functions():
    text = (ROOT / "include" / "intspmv.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text)
    skip = {"if", "for", "while", "return", "sizeof", "defined"}
    protos = set()
    for m in re.finditer(r"^[A-Za-z_][^;{}#]*?\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;]*\)\s*;", text, flags=re.M | re.S):
        if m.group(1) not in skip:
            protos.add(m.group(1))
    assert protos, names
    return sorted(protos)


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python prototype table covers the same set
    assert set(declared_functions()) <= set(abi.PROTOTYPES), set(declared_functions()) - set(abi.PROTOTYPES)
    load()  # binds every prototype


def test_struct_sizes_match_reference():
    from oracle import Reference
    mine = [C.sizeof(t) for t in (abi.StrMatCSR, abi.StrFormatData, abi.StrErr, abi.StrRes, abi.StrMatAXC,
                                  abi.StrMatK1, abi.StrMatAXT)]
    assert mine == [96, 48, 24, 80, 32, 56, 72]
    if Reference.available():
        assert mine == [Reference().sizeof(i) for i in range(7)]


def test_status_strings():
    lib = load()
    for st in range(7):
        assert lib.ispmv_status_string(st)
    assert b"unknown" in lib.ispmv_status_string(99)


@pytest.mark.parametrize("ext", [".csr", ".bin"])
@pytest.mark.parametrize("name", ["random257_empty", "long_rows_700", "one_by_one"])
def test_file_round_trip(tmp_path, ext, name):
    g = load_golden(name)
    c = F.CSR(g["row"], g["col"], g["val"])
    p = tmp_path / f"m{ext}"
    c.write(str(p))
    d = F.CSR.read(str(p))
    assert np.array_equal(d.row, c.row) and np.array_equal(d.col, c.col)
    assert np.array_equal(d.val, c.val)  # %.17g text keeps every bit
    assert np.array_equal(d.rl[:d.n], g["rl"])


def test_bin_layout_is_the_reference_one(tmp_path):
    """u32 n, u32 nnz, f64 val[nnz], u32 col[nnz], u32 row[n+1]."""
    g = load_golden("poisson8")
    n, nnz = len(g["row"]) - 1, len(g["col"])
    p = tmp_path / "m.bin"
    with open(p, "wb") as f:
        f.write(np.array([n, nnz], np.uint32).tobytes())
        f.write(g["val"].astype(np.float64).tobytes())
        f.write(g["col"].astype(np.uint32).tobytes())
        f.write(g["row"].astype(np.uint32).tobytes())
    d = F.CSR.read(str(p))
    assert np.array_equal(d.col, g["col"]) and np.array_equal(d.val, g["val"])


def test_malformed_files_are_errors(tmp_path):
    p = tmp_path / "bad.bin"
    p.write_bytes(np.array([10, 5], np.uint32).tobytes() + b"\x00" * 7)  # short read
    with pytest.raises(IntSpmvError):
        F.CSR.read(str(p))
    q = tmp_path / "bad.csr"
    q.write_text("3 2\n1.0 0\n2.0 7\n0 1 2 2\n")  # column out of range
    with pytest.raises(IntSpmvError):
        F.CSR.read(str(q))
    with pytest.raises(IntSpmvError):
        F.CSR.read(str(tmp_path / "m.mtx"))  # neither .csr nor .bin


@pytest.mark.parametrize("name", golden_names())
def test_sta_report_matches_reference(tmp_path, name):
    g = load_golden(name)
    c = F.CSR(g["row"], g["col"], g["val"])
    path = tmp_path / "dir.with.dots" / "m.csr"
    path.parent.mkdir()
    load().printMatrixStats(str(path).encode(), C.byref(c.c))
    mine = (path.parent / "m.sta").read_text().splitlines()
    ref = str(g["sta"]).splitlines()
    assert len(mine) == len(ref)
    for a, b in zip(mine, ref):
        if a.startswith("name:"):
            continue  # the file name itself differs
        assert a == b


def test_plan_layout_struct_matches_header():
    """ispmv_plan_layout's C layout (six u64 lengths, val_bytes, spl, then
    the window count) as the ctypes mirror declares it: 64 bytes, nwin last
    at offset 56."""
    assert C.sizeof(abi.PlanLayout) == 64
    assert abi.PlanLayout.nwin.offset == 56


def test_plan_from_device_csr_checks_shapes_before_any_device_call():
    """Plan.from_device_csr rejects inconsistent array lengths and a
    non-FP64 value array on the host, before the library is called."""
    import torch

    from int_spmv_b200 import device as D
    row = torch.tensor([0, 1, 2], dtype=torch.int32)
    col = torch.tensor([0, 1], dtype=torch.int32)
    with pytest.raises(ValueError):
        D.Plan.from_device_csr(row, col, torch.zeros(3, dtype=torch.float64))
    with pytest.raises(ValueError):
        D.Plan.from_device_csr(row, col, torch.zeros(2, dtype=torch.float32))
    with pytest.raises(ValueError):
        D.Plan.from_device_csr(torch.tensor([0], dtype=torch.int32), col[:0], torch.zeros(0, dtype=torch.float64))


def test_k1_entry_points_reject_null_arrays_before_any_device_call():
    """The device K1 entry points check their arrays on the host: a null
    value or column array is ISPMV_ERR_ARG, returned before anything is
    launched (so this needs no GPU).  Any non-null address passes the check,
    which is all these calls read before returning."""
    lib = load()
    p = C.c_void_p(16)  # never dereferenced: the null check fails first
    nul = C.c_void_p(0)
    assert lib.ispmv_dev_k1_spmv_noalloc(16, 2, nul, p, p, p, p, p, p, None) == 1
    assert lib.ispmv_dev_k1_spmv_noalloc(16, 2, p, nul, p, p, p, p, p, None) == 1
    assert lib.ispmv_dev_int_k1(2, nul, p, p, p, p, p, None) == 1
    assert lib.ispmv_dev_int_k1(2, p, nul, p, p, p, p, None) == 1
    assert lib.ispmv_dev_int_k1p(0xFF, 2, nul, p, p, p, p, p, p, None) == 1
    assert lib.ispmv_dev_int_k1p(0xFF, 2, p, nul, p, p, p, p, p, None) == 1


def test_time_main_rejects_bad_arguments_before_any_device_call():
    """ispmv_plan_time_main checks its arguments on the host: a null plan,
    x, y or result pointer, or fewer than one repetition, is ISPMV_ERR_ARG,
    returned before any event is made or kernel launched (no GPU needed)."""
    lib = load()
    p = C.c_void_p(16)  # never dereferenced: an argument check fails first
    nul = C.c_void_p(0)
    ms = C.c_double()
    assert lib.ispmv_plan_time_main(nul, p, p, 1, None, C.byref(ms)) == 1
    assert lib.ispmv_plan_time_main(p, nul, p, 1, None, C.byref(ms)) == 1
    assert lib.ispmv_plan_time_main(p, p, nul, 1, None, C.byref(ms)) == 1
    assert lib.ispmv_plan_time_main(p, p, p, 0, None, C.byref(ms)) == 1
    assert lib.ispmv_plan_time_main(p, p, p, 1, None, None) == 1
