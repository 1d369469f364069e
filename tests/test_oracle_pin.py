"""The oracle (oracle/oracle.c, the C restatement) is pinned here against the
reference's own outputs: the golden fixtures made by the reference build
(tests/golden/make_golden.py) and, where oracle/_ref is present, fresh runs
of the reference on new seeded inputs."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_names, load_golden
from int_spmv_b200 import matrices as M
from oracle import Oracle, Reference

AXT_CASES = [("NOC", 1, 128), ("NOC", 4, 128), ("NOC", 8, 128), ("NOC", 16, 128), ("NOC", 48, 128), ("NOC", 3, 128),
             ("COM", 1, 128), ("COM", 1, 256), ("COM", 1, 512), ("COM", 1, 8)]


@pytest.fixture(scope="module")
def orc():
    return Oracle()


def _close(a, b, rtol=1e-13):
    scale = max(1.0, float(np.abs(b).max(initial=0.0)))
    return float(np.abs(a - b).max(initial=0.0)) <= rtol * scale


@pytest.mark.parametrize("name", golden_names())
def test_oracle_stats_and_csr(orc, name):
    g = load_golden(name)
    st = orc.stats(g["row"], g["col"])
    assert np.array_equal(st["rl"], g["rl"])
    assert [st["rmin"], st["rave"], st["rmax"], st["rsd"], st["bw"]] == list(g["stats"])
    assert np.array_equal(orc.cf_csr(g["row"], g["col"], g["val"], g["x"]), g["y_csr"])  # bit-exact


@pytest.mark.parametrize("name", golden_names())
def test_oracle_axc_k1(orc, name):
    g = load_golden(name)
    a = orc.axc(g["row"], g["col"], g["val"], g["x"], g["rl"])
    assert np.array_equal(a["brp"], g["axc_brp"]) and np.array_equal(a["ax"], g["axc_ax"])
    assert np.array_equal(orc.axc_spmv(a["ax"], a["brp"]), g["y_axc"])
    k = orc.k1(g["row"], g["col"], g["val"], g["rl"])
    for f in ("permi", "nmc", "chp", "val", "col"):
        assert np.array_equal(k[f], g["k1_" + f]), f
    n = len(g["rl"])
    res = orc.k1_spmv(k, g["x"])
    assert np.array_equal(res, g["k1_res"])
    assert np.array_equal(orc.k1_order(k["permi"], res, n), g["y_k1"])
    assert np.array_equal(orc.k1p_spmv(k, g["x"], n), g["y_k1p"])


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("mode,th,bs", AXT_CASES)
def test_oracle_axt(orc, name, mode, th, bs):
    g = load_golden(name)
    key = f"axt_{mode}_{th}_{bs}"
    t = orc.axt(g["row"], g["col"], g["val"], g["x"], g["rl"], 8, th, mode, bs)
    assert np.array_equal(t["con"], g[key + "_con"])
    assert np.array_equal(t["ax"], g[key + "_ax"])
    assert np.array_equal(t["sec"], g[key + "_sec"])
    meta = g[key + "_meta"]
    assert [t["tileN"], t["lenAX"], t["lenSEC"]] == list(meta[:3])
    if mode == "COM":
        assert t["log"] == meta[4]
    n = len(g["rl"])
    if mode == "COM":
        y = orc.axt_com_h1_ref(bs, t["log"], t["tileN"], t["lenSEC"], t["ax"], t["sec"], n)
        assert np.array_equal(y, g["y_" + key])  # the reference's result, defects included
    elif th == 1:
        assert np.array_equal(orc.axt_noc_h1_spmv(t["tileN"], t["ax"], t["sec"], n), g["y_" + key])
    else:
        # the reference adds each tile's 8 lane sums from a nested OpenMP region: order varies
        assert _close(orc.axt_noc_spmv(t["tileN"], th, t["ax"], t["sec"], n), g["y_" + key])


@pytest.mark.parametrize("name", golden_names())
def test_oracle_errors(orc, name):
    g = load_golden(name)
    a, r, p = orc.get_errors(g["y_csr"], g["y_axc"])
    ga, gr, gp = g["errors_axc"]
    assert a == ga and p == gp and (r == gr or (np.isnan(r) and np.isnan(gr)))


def test_com_defect_reproduced(orc):
    """Row-0 segments whose descriptor is 0 are dropped by the reference's
    compacted kernel (README.md:33): the golden y shows it, the CSR y not."""
    g = load_golden("one_by_one")
    assert g["y_axt_COM_1_128"][0] == 0.0 and g["y_csr"][0] != 0.0
    g = load_golden("row0_129")
    assert abs(g["y_axt_COM_1_128"][0] - g["y_csr"][0]) > 1e-6


needs_ref = pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built on this host")


@needs_ref
@pytest.mark.parametrize("seed", [101, 102])
def test_oracle_vs_live_reference(orc, seed):
    R = Reference()
    row, col, val = M.random_csr(611, seed, rl_max=90, empty_frac=0.05)
    n = 611
    x = M.uniform_x(n, seed)
    s = R.csr(row, col, val)
    s._keep[3][:] = np.diff(row)
    assert np.array_equal(R.cf_csr(s, x), orc.cf_csr(row, col, val, x))
    rl = np.diff(row).astype(np.uint32)
    for mode, th, bs in AXT_CASES:
        t = R.build_axt(s, x, 8, th, mode, bs)
        o = orc.axt(row, col, val, x, rl, 8, th, mode, bs)
        for f in ("con", "ax", "sec"):
            assert np.array_equal(t[f], o[f]), (mode, th, bs, f)
        R.free_axt(t)
    k = R.build_k1(s, x)
    ok = orc.k1(row, col, val, rl)
    for f in ("permi", "nmc", "chp", "val", "col"):
        assert np.array_equal(k[f], ok[f])
    R.free_k1(k)
