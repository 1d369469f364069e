"""The autotuner's host side, without a GPU: the matrix signature its cache
is keyed by, and a cached choice returned before any candidate is timed."""
from __future__ import annotations

import json

import numpy as np

from int_spmv_b200 import autotune as T
from int_spmv_b200 import formats as F
from int_spmv_b200 import matrices as M


def _csr(n=5000, seed=7):
    row, col, val = M.random_csr(n, seed, rl_max=40, empty_frac=0.05)
    return F.CSR(row, col, val)


def test_signature_is_deterministic_and_keyed_by_form():
    a, b = _csr(), _csr()
    s = T.signature(a)
    assert s == T.signature(b)  # the same matrix, built twice
    assert len(s) == 16
    assert T.signature(a, val="f32") != s
    assert T.signature(a, col="d16") != s
    assert T.signature(a, k=8) != s and T.signature(a, k=8) != T.signature(a, k=16)
    # a matrix of another shape (longer rows) has another signature
    row, col, val = M.random_csr(5000, 7, rl_max=400, empty_frac=0.0)
    assert T.signature(F.CSR(row, col, val)) != s


def test_cached_choice_is_returned_without_timing(tmp_path, monkeypatch):
    cache = tmp_path / "tune.json"
    monkeypatch.setenv("ISPMV_TUNE_CACHE", str(cache))
    csr = _csr()
    sig = T.signature(csr, "f64", "u32", None)
    choice = {"format": "COM128", "kwargs": {"kernel": "wide", "variant": 26}, "seconds": 1e-4, "when": 0.0,
              "timings": []}
    cache.write_text(json.dumps({sig: choice}))

    def no_timing(*a, **k):  # a cache hit must not time any candidate
        raise AssertionError("a candidate was timed")

    monkeypatch.setattr(T, "_time", no_timing)
    monkeypatch.setattr(T, "build_plan", no_timing)
    got = T.tune(csr, np.zeros(csr.n))
    assert got["cached"] is True and got["signature"] == sig
    assert got["format"] == "COM128" and got["kwargs"] == {"kernel": "wide", "variant": 26}


def test_cache_store_round_trip(tmp_path, monkeypatch):
    cache = tmp_path / "sub" / "tune.json"
    monkeypatch.setenv("ISPMV_TUNE_CACHE", str(cache))
    assert T.cache_path() == cache
    assert T._load_cache() == {}  # no file yet
    T._store_cache({"abc": {"format": "CSR", "kwargs": {}}})
    assert T._load_cache() == {"abc": {"format": "CSR", "kwargs": {}}}
    cache.write_text("not json")
    assert T._load_cache() == {}  # a damaged cache is ignored, not fatal
