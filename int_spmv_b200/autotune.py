"""Per-matrix autotuner for the plans.

For a matrix it times candidate plans on the current GPU and keeps the
fastest.  The candidates vary:
- the format: AXT compacted, AXT tileHeight 1, 4, 8 or 16, AXC, CSR, K1;
- the kernel family: lane-interleaved slot stream (stream_wide), slot stream
  with plain loads or bulk-copy staging, tile columns, or row-parallel;
- the kernel variant: slots per lane (the vector width: 8 or 16 for
  stream_wide, 2 or 4 for stream_ldg), prefetch depth or bulk-copy stages,
  warps per SM (threads per tile) and a per-CTA x window in shared memory;
- the segment size;
- for SpMM, the right-hand sides per pass (the RHS block).

Choices are cached per matrix signature in a JSON file, so a second plan for
a matrix of the same shape reuses the choice without timing.  The signature
is the size, the row-length histogram, the bandwidth and the share of
near-diagonal columns.

The cache file is $ISPMV_TUNE_CACHE, else ~/.cache/int_spmv_b200/tune.json.
"""
from __future__ import annotations

import hashlib
import json
import os
import time
from pathlib import Path

import numpy as np

from .formats import CSR

# (format, plan keyword arguments)
SPMV_CANDIDATES = [
    ("COM128", dict(kernel="wide", variant=0)),   # 16 slots per lane
    ("COM128", dict(kernel="wide", variant=4)),   # 8 slots per lane
    ("COM128", dict(kernel="wide", variant=8)),   # 16 slots per lane, 8192-slot segments
    ("COM128", dict(kernel="wide", variant=9)),   # 16 slots per lane, 2048-slot segments
    ("COM128", dict(kernel="wide", variant=11)),  # bulk-copy staged, 16 slots per lane
    ("COM128", dict(kernel="wide", variant=16)),  # 8 slots per lane, x gathered through the texture pipe
    ("COM128", dict(kernel="wide", variant=26)),  # 8 slots per lane, per-CTA x window by one bulk copy
    ("COM128", dict(kernel="wide", variant=32)),  # 8 slots per lane, next batch's columns loaded ahead
    ("NOC1", dict(kernel="wide", variant=0)),
    ("NOC4", dict()),                             # tile columns as a lane-interleaved stream (AUTO variant)
    ("NOC8", dict()),
    ("CSR", dict()),                              # CSR order as a lane-interleaved stream (AUTO variant)
    ("AXC", dict()),                              # the brick stream, lane-interleaved (AUTO variant)
    ("COM128", dict(kernel="ldg", variant=0)),
    ("COM128", dict(kernel="ldg", variant=2)),
    ("COM128", dict(kernel="ldg", variant=12)),
    ("COM128", dict(kernel="tma", variant=0)),
    ("COM128", dict(kernel="ldg", variant=2, units_per_warp=1024)),
    ("NOC1", dict(kernel="ldg", variant=2)),
    ("NOC4", dict(kernel="ldg")),
    ("NOC8", dict(kernel="tma")),
    ("CSR", dict(kernel="rows")),
    ("AXC", dict(kernel="rows")),
    ("K1P", dict()),
]
# SpMM: plan kernel x columns per pass x four ("wide") or two ("ldg") columns per lane
SPMM_CANDIDATES = [(fmt, dict(kw, rhs_block=b, spmm_kernel=sk))
                   for fmt, kw in (("COM128", dict(kernel="ldg")), ("NOC1", dict(kernel="ldg")),
                                   ("COM128", dict(kernel="wide", variant=4)))
                   for b in (8, 16, 32) for sk in ("wide", "ldg")]


def cache_path() -> Path:
    p = os.environ.get("ISPMV_TUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "int_spmv_b200" / "tune.json"


def signature(csr: CSR, val: str = "f64", col: str = "u32", k: int | None = None) -> str:
    """Shape of the matrix that the kernel choice depends on."""
    n, nnz = csr.n, csr.nnz
    rl = csr.rl[:n].astype(np.int64)
    hist = np.bincount(np.minimum(np.log2(np.maximum(rl, 1)).astype(np.int64), 16), minlength=17)
    hist = np.round(hist / max(n, 1), 2).tolist()
    rows = np.repeat(np.arange(n, dtype=np.int64), rl)
    sample = slice(None, None, max(1, nnz // 200000))
    d = np.abs(csr.col[sample].astype(np.int64) - rows[sample])
    near = round(float(np.mean(d <= 1024)) if d.size else 1.0, 2)
    key = dict(n=int(round(n, -int(max(0, np.log10(max(n, 1)) - 2)))), mean_rl=round(nnz / max(n, 1), 1),
               hist=hist, bw=round(csr.stats()["bw"] / max(n, 1), 2), near=near, val=val, col=col, k=k)
    return hashlib.sha1(json.dumps(key, sort_keys=True).encode()).hexdigest()[:16]


def _load_cache() -> dict:
    try:
        return json.loads(cache_path().read_text())
    except Exception:
        return {}


def _store_cache(c: dict) -> None:
    p = cache_path()
    p.parent.mkdir(parents=True, exist_ok=True)
    tmp = p.with_suffix(".tmp")
    tmp.write_text(json.dumps(c, indent=1, sort_keys=True))
    tmp.replace(p)


def build_plan(csr: CSR, x, fmt: str, val: str = "f64", col: str = "u32", **kw):
    """The plan of one candidate (format name as in SPMV_CANDIDATES)."""
    from . import device as D
    from . import formats as F
    if fmt == "CSR":
        return D.Plan(csr, None, val=val, col=col, **kw)
    if fmt == "AXC":
        return D.Plan(csr, F.getFormatDataAXC(0, csr, x)[1], val=val, col=col, **kw)
    if fmt in ("K1", "K1P"):
        return D.Plan(csr, F.getFormatDataK1(8, csr, x)[1], reorder=fmt == "K1P", val=val, col=col, **kw)
    if fmt.startswith("NOC"):
        return D.Plan(csr, F.getFormatDataAXT(0, 128, 8, int(fmt[3:]), "NOC", csr, x)[1], val=val, col=col, **kw)
    if fmt.startswith("COM"):
        return D.Plan(csr, F.getFormatDataAXT(0, int(fmt[3:]), 8, 1, "COM", csr, x)[1], val=val, col=col, **kw)
    raise ValueError(fmt)


def _time(fn, reps: int) -> float:
    import torch
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps * 1e-3


def tune(csr: CSR, x=None, val: str = "f64", col: str = "u32", k: int | None = None, candidates=None,
         reps: int = 30, use_cache: bool = True, verbose: bool = False) -> dict:
    """Times the candidates (SpMV, or SpMM with k right-hand sides) and
    returns {"format", "kwargs", "seconds", "signature", "timings"}."""
    import torch
    sig = signature(csr, val, col, k)
    cache = _load_cache() if use_cache else {}
    if sig in cache:
        return dict(cache[sig], signature=sig, cached=True)
    cands = candidates or (SPMM_CANDIDATES if k else SPMV_CANDIDATES)
    x = np.zeros(csr.n) if x is None else x
    dev_x = torch.from_numpy(np.random.default_rng(0).uniform(-1, 1, (csr.n, k) if k else csr.n)).cuda()
    out = torch.empty_like(dev_x)
    timings = []
    for fmt, kw in cands:
        try:
            p = build_plan(csr, x, fmt, val, col, **kw)
            t = _time((lambda: p.spmm(dev_x, out)) if k else (lambda: p.spmv(dev_x, out)), reps)
            del p
        except Exception as e:  # a candidate the matrix cannot use (e.g. a form the path lacks)
            if verbose:
                print(f"tune: {fmt} {kw} skipped: {e}")
            continue
        timings.append((t, fmt, kw))
        if verbose:
            print(f"tune: {fmt} {kw} {t * 1e3:.4f} ms")
    if not timings:
        raise RuntimeError("autotune: no candidate plan could be built")
    timings.sort(key=lambda r: r[0])
    t, fmt, kw = timings[0]
    choice = dict(format=fmt, kwargs=kw, seconds=t, when=time.time(),
                  timings=[dict(format=f, kwargs=w, seconds=s) for s, f, w in timings])
    if use_cache:
        cache[sig] = choice
        _store_cache(cache)
    return dict(choice, signature=sig, cached=False)


def best_plan(csr: CSR, x=None, val: str = "f64", col: str = "u32", k: int | None = None, **tune_kw):
    """(plan, choice): the fastest plan for this matrix (cached per signature)."""
    choice = tune(csr, x, val, col, k, **tune_kw)
    x = np.zeros(csr.n) if x is None else x
    return build_plan(csr, x, choice["format"], val, col, **choice["kwargs"]), choice
