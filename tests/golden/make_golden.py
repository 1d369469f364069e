"""Generates tests/golden/*.npz: outputs of the reference itself
(edoardoCB/int_spmv intSpmv_main.c, compiled from its own source by
oracle/Makefile into oracle/_ref) on small seeded matrices covering the edge
cases the format rules have.  The reference ships no tests or fixtures, so
these are its known answers.

    python tests/golden/make_golden.py      (needs oracle/_ref, AVX-512)

Each fixture holds the input CSR and x, the reference's row statistics,
every builder's arrays and struct fields, and every reference kernel's y
(one OpenMP thread, so the accumulating kernels add in tile order).
"""
from __future__ import annotations

import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from int_spmv_b200 import matrices as M  # noqa: E402
from oracle import Reference, build  # noqa: E402

OUT = Path(__file__).resolve().parent
U32 = np.uint32

AXT_CASES = [("NOC", 1, 128), ("NOC", 4, 128), ("NOC", 8, 128), ("NOC", 16, 128), ("NOC", 48, 128), ("NOC", 3, 128),
             ("COM", 1, 128), ("COM", 1, 256), ("COM", 1, 512), ("COM", 1, 8)]


def _csr_from_lists(n, rows):
    row = np.zeros(n + 1, np.int64)
    row[1:] = np.cumsum([len(r) for r in rows])
    col = np.concatenate([np.asarray(r, np.int64) for r in rows]) if row[-1] else np.zeros(0, np.int64)
    return row.astype(U32), col.astype(U32)


def cases():
    rng = np.random.default_rng(2024)
    out = {}
    r, c, v = M.poisson2d(8)
    out["poisson8"] = (r, c, v)
    out["random257_empty"] = M.random_csr(257, 11, rl_max=40, empty_frac=0.15)
    # single row of length 1: row 0's descriptor encodes as 0 (compacted AXT)
    out["one_by_one"] = (np.array([0, 1], U32), np.array([0], U32), np.array([2.5]))
    # row 0 of length 129 crosses a 128-slot block boundary with a 1-slot remainder
    rows = [sorted(rng.choice(200, 129, replace=False))] + [sorted(rng.choice(200, int(k), replace=False))
                                                           for k in rng.integers(0, 30, 199)]
    r, c = _csr_from_lists(200, rows)
    out["row0_129"] = (r, c, rng.standard_normal(len(c)))
    # equal row lengths: every K1 sort key ties
    rows = [sorted(rng.choice(100, 5, replace=False)) for _ in range(100)]
    r, c = _csr_from_lists(100, rows)
    out["ties100"] = (r, c, rng.standard_normal(len(c)))
    # n not a multiple of 8, rows longer than 512
    rows = [sorted(rng.choice(700, int(k), replace=False)) for k in [600, 3, 0, 513, 17, 1, 0, 64, 9, 700, 2, 0, 31]]
    # the long rows need n >= 700 distinct columns: 13 such rows, then 687 empty ones
    rows13 = rows + [[] for _ in range(700 - 13)]
    r, c = _csr_from_lists(700, rows13)
    out["long_rows_700"] = (r, c, rng.standard_normal(len(c)))
    # mostly empty
    rows = [[] for _ in range(37)]
    rows[5] = [0, 3, 36]
    rows[36] = [36]
    r, c = _csr_from_lists(37, rows)
    out["mostly_empty37"] = (r, c, rng.standard_normal(len(c)))
    return out


def main() -> None:
    build()
    R = Reference()
    assert R.num_ite() == 1
    tmp = Path(tempfile.mkdtemp(prefix="ispmvgolden"))
    for name, (row, col, val) in cases().items():
        row, col, val = np.asarray(row, U32), np.asarray(col, U32), np.asarray(val, np.float64)
        n = len(row) - 1
        x = M.uniform_x(n, 7)
        s = R.csr(row, col, val)
        st = R.stats(tmp / "m.csr", s)
        sta = (tmp / "m.sta").read_text()
        d = dict(row=row, col=col, val=val, x=x, rl=st["rl"],
                 stats=np.array([st["rmin"], st["rave"], st["rmax"], st["rsd"], st["bw"]], np.float64),
                 sta=np.array(sta), y_csr=R.cf_csr(s, x))
        a = R.build_axc(s, x)
        d.update(axc_brp=a["brp"], axc_ax=a["ax"], axc_fd=np.array([a["fd"][1], a["fd"][2]]),
                 y_axc=R.int_axc(a, n))
        R.free_axc(a)
        k = R.build_k1(s, x)
        res, y = R.int_k1(k, x, n)
        d.update(k1_permi=k["permi"], k1_nmc=k["nmc"], k1_chp=k["chp"], k1_val=k["val"], k1_col=k["col"],
                 k1_fd=np.array([k["fd"][1], k["fd"][2]]), k1_res=res, y_k1=y, y_k1p=R.int_k1p(k, x, n),
                 k1_mask=np.array(R.lib.ref_k1p_mask_of(__import__("ctypes").byref(k["struct"]))))
        R.free_k1(k)
        for mode, th, bs in AXT_CASES:
            t = R.build_axt(s, x, 8, th, mode, bs)
            key = f"axt_{mode}_{th}_{bs}"
            d[key + "_con"], d[key + "_ax"], d[key + "_sec"] = t["con"], t["ax"], t["sec"]
            d[key + "_meta"] = np.array([t["tileN"], t["lenAX"], t["lenSEC"], t["lenCON"], t["log"], t["logTH"]],
                                        np.int64)
            d[key + "_fd"] = np.array([t["fd"][1], t["fd"][2]])
            d[key + "_name"] = np.array(t["fd"][0])
            d["y_" + key] = R.int_axt(t, n, bs=bs)
            R.free_axt(t)
        d["errors_axc"] = np.array(R.get_errors(d["y_csr"], d["y_axc"]))
        np.savez_compressed(OUT / f"{name}.npz", **d)
        print(name, n, len(col))


if __name__ == "__main__":
    main()
