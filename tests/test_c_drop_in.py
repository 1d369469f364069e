"""The drop-in from C: tests/c/drop_in.c, the reference's driver
(intSpmv_main.c:1617-1761) written against include/intspmv.h, is compiled
and linked with libintspmv.so in the reference's two configurations,
FP_TYPE=FP_DOUBLE and FP_TYPE=FP_FLOAT.

On the CPU: both link, and the FP32 build binds the `_f32` symbols.
On the GPU: both run on golden matrices; every kernel's y (written by the
program) is at parity with the oracle's FP64 CSR product on the same
inputs (FP64: 1e-12 (|A||x|)_i; FP32: values and x rounded to FP32, then
1e-6 (|A||x|)_i), and the test_* harness rows carry the reference's names,
positive times and the errors of each kernel against cf_CSR.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, load_golden
from paritylib import TOL_F32, TOL_F64, assert_parity

SRC = ROOT / "tests" / "c" / "drop_in.c"
LIBDIR = ROOT / "int_spmv_b200"
KERNELS = ["cf_CSR", "int_AXC", "int_k1", "int_k1p", "int_axt_noc_h1_hw8", "int_axt_noc_h4_hw8", "int_axt_noc_h8_hw8",
           "int_axt_com_h1_hw8_bs128", "int_axt_com_h1_hw8_bs256", "int_axt_com_h1_hw8_bs512"]
DUMPS = ["cf_CSR", "int_axc", "int_k1", "int_k1p", "int_axt_noc_h1_hw8", "int_axt_noc_h4_hw8", "int_axt_noc_h8_hw8",
         "int_axt_com_h1_hw8_bs128", "int_axt_com_h1_hw8_bs256", "int_axt_com_h1_hw8_bs512"]


def _compile(out: Path, fp32: bool) -> Path:
    exe = out / ("drop_in_f32" if fp32 else "drop_in_f64")
    cmd = ["gcc", "-O2", "-std=gnu11", "-Wall", "-Werror", f"-I{ROOT / 'include'}", str(SRC), "-o", str(exe),
           f"-L{LIBDIR}", "-lintspmv", f"-Wl,-rpath,{LIBDIR}"]
    if fp32:
        cmd.insert(1, "-DFP_TYPE=FP_FLOAT")
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.fixture(scope="module")
def exes(tmp_path_factory):
    d = tmp_path_factory.mktemp("drop_in")
    return {False: _compile(d, False), True: _compile(d, True)}


def _undefined(exe: Path) -> set[str]:
    r = subprocess.run(["nm", "-u", str(exe)], capture_output=True, text=True, check=True)
    return {line.split()[-1].split("@")[0] for line in r.stdout.splitlines() if line.strip()}


def test_both_configurations_link(exes):
    """FP_TYPE=FP_FLOAT resolves every reference name to its `_f32` symbol;
    the default build binds the FP64 names."""
    u64, u32 = _undefined(exes[False]), _undefined(exes[True])
    names = {"matrixReading", "getFormatDataAXT", "cf_CSR", "int_axt_com_h1", "test_int_k1", "initVec"}
    assert names <= u64
    assert not (names & u32)
    assert {n + "_f32" for n in names} <= u32


def _table(text: str) -> dict:
    rows = {}
    lines = text.splitlines()
    start = next(i for i, line in enumerate(lines) if line.startswith("kernels' results"))
    for line in lines[start + 2:]:
        f = line.split()
        if len(f) == 7:
            rows[f[0]] = dict(et=float(f[1]), gflops=float(f[2]), ot=float(f[3]), aErr=float(f[4]),
                              rErr=float(f[5]), pos=int(f[6]))
    return rows


@pytest.mark.gpu
@pytest.mark.parametrize("fp32", [False, True])
@pytest.mark.parametrize("case", ["random257_empty", "long_rows_700", "row0_129", "poisson64"])
def test_drop_in_runs_at_parity(exes, tmp_path, fp32, case):
    from int_spmv_b200 import formats as F
    from int_spmv_b200 import matrices as M
    from oracle import Oracle
    if case == "poisson64":
        row, col, val = M.poisson2d(64)
    else:
        g = load_golden(case)
        row, col, val = g["row"], g["col"], g["val"]
    path = tmp_path / f"{case}.csr"
    F.CSR(row, col, val).write(str(path))
    out = tmp_path / "y"
    out.mkdir()
    env = dict(os.environ, ISPMV_NUM_ITE="3")
    r = subprocess.run([str(exes[fp32]), str(path), str(out)], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert ("FPT: float" if fp32 else "FPT: double") in r.stdout
    n = len(row) - 1
    x = np.arange(n, dtype=np.float64)  # initVec, M:361-367 (exact in FP32 at these sizes)
    v = val.astype(np.float32).astype(np.float64) if fp32 else val
    orc = Oracle()
    yref, absax = orc.cf_csr(row, col, v, x), orc.abs_csr(row, col, v, x)
    tol = TOL_F32 if fp32 else TOL_F64
    dt = np.float32 if fp32 else np.float64
    for name in DUMPS:
        y = np.fromfile(out / f"{name}.y", dtype=dt).astype(np.float64)
        assert len(y) == n, name
        assert_parity(y, yref, absax, tol, what=f"{'FP32' if fp32 else 'FP64'} {name} on {case}")
    t = _table(r.stdout)
    assert list(t) == KERNELS, list(t)
    for name, row_ in t.items():
        assert row_["et"] > 0 and row_["gflops"] > 0, name
        assert row_["rErr"] <= (1e-6 if fp32 else 1e-12), (name, row_)
    assert t["int_k1"]["ot"] > 0 and all(t[k]["ot"] == 0 for k in KERNELS if k != "int_k1")
