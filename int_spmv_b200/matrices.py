"""Seeded synthetic matrices of the benchmark workloads (numpy, host side).

The reference (edoardoCB/int_spmv) reads matrices from files
(intSpmv_main.c:187-249) and its job scripts name two public matrices
(MDE.csr, M25_Serena.bin) that are not available here; these generators stand
in for them with the workloads' stated shapes, sizes and value distributions.
All return CSR arrays: row (u32, n+1), col (u32, nnz), val (f64, nnz), with
columns ascending inside each row.
"""
from __future__ import annotations

import numpy as np

U32 = np.uint32


def _csr_from_sorted_keys(n: int, keys: np.ndarray, vals: np.ndarray):
    rows = (keys // n).astype(np.int64)
    cols = (keys % n).astype(U32)
    counts = np.bincount(rows, minlength=n)
    row = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=row[1:])
    return row.astype(U32), cols, vals


def poisson2d(m: int):
    """2D 5-point Laplacian on an m x m grid, natural row-major order:
    4.0 on the diagonal, -1.0 to the 4 neighbours.  n = m^2,
    nnz = 5n - 4m."""
    n = m * m
    offs = [(-m, -1.0), (-1, -1.0), (0, 4.0), (1, -1.0), (m, -1.0)]  # ascending column offsets
    idx = np.arange(n, dtype=np.int64)
    x, yv = idx % m, idx // m
    valid = np.stack([yv > 0, x > 0, np.ones(n, bool), x < m - 1, yv < m - 1], axis=1)
    return _stencil_fill(n, idx, valid, [o for o, _ in offs], lambda k, cnt: np.full(cnt, offs[k][1]))


def _stencil_fill(n, idx, valid, offsets, value_of):
    counts = valid.sum(axis=1)
    row = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=row[1:])
    pos = np.cumsum(valid, axis=1, dtype=np.int16) - 1
    nnz = int(row[-1])
    col = np.empty(nnz, dtype=U32)
    val = np.empty(nnz, dtype=np.float64)
    for k, o in enumerate(offsets):
        sel = valid[:, k]
        r = idx[sel]
        dst = row[r] + pos[sel, k]
        col[dst] = (r + o).astype(U32)
        val[dst] = value_of(k, int(sel.sum()))
    return row.astype(U32), col, val


def stencil27(m: int, seed: int = 2):
    """3D 27-point stencil on an m^3 grid, natural order: 26.0 on the
    diagonal, -1.0 + U[-0.1, 0.1] off it (numpy default_rng(seed), drawn per
    neighbour offset in ascending column order).  nnz = (3m-2)^3."""
    n = m ** 3
    rng = np.random.default_rng(seed)
    idx = np.arange(n, dtype=np.int64)
    x, y, z = idx % m, (idx // m) % m, idx // (m * m)
    offsets, valid = [], []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                offsets.append(dz * m * m + dy * m + dx)
                v = np.ones(n, bool)
                if dx == -1: v &= x > 0
                if dx == 1: v &= x < m - 1
                if dy == -1: v &= y > 0
                if dy == 1: v &= y < m - 1
                if dz == -1: v &= z > 0
                if dz == 1: v &= z < m - 1
                valid.append(v)
    valid = np.stack(valid, axis=1)
    diag = offsets.index(0)

    def value_of(k, cnt):
        if k == diag:
            return np.full(cnt, 26.0)
        return -1.0 + rng.uniform(-0.1, 0.1, cnt)

    return _stencil_fill(n, idx, valid, offsets, value_of)


def powerlaw(n: int, seed: int = 1, mu: float = 2.2, sigma: float = 1.0, rl_min: int = 1, rl_max: int = 5000,
             band: int = 1000, band_frac: float = 0.7):
    """Power-law (lognormal) row lengths: rl = clip(rint(lognormal(mu,
    sigma)), rl_min, rl_max).  Of each row's rl columns, rint(band_frac*rl)
    are uniform in the window [r-band, r+band] clipped to [0, n) and the rest
    uniform over [0, n); a column drawn twice in a row is kept once (a band
    draw before a uniform one) and the lost draw is redrawn from its own
    distribution until every row has rl distinct columns.  Values N(0,1).
    numpy default_rng(seed) drives everything, in this order: row lengths,
    then per round the band columns and the uniform columns; values last."""
    rng = np.random.default_rng(seed)
    rl = np.clip(np.rint(rng.lognormal(mu, sigma, n)), rl_min, min(rl_max, n)).astype(np.int64)
    r_all = np.arange(n, dtype=np.int64)
    win = np.minimum(r_all + band, n - 1) - np.maximum(r_all - band, 0) + 1
    nb = np.minimum(np.rint(band_frac * rl).astype(np.int64), win)
    need_b, need_r = nb, rl - nb
    accepted = None  # sorted int64 keys row*n + col
    extra = np.empty(0, np.int64)
    for _ in range(64):
        if not need_b.any() and not need_r.any():
            break
        rb = np.repeat(r_all, need_b)
        lo = np.maximum(rb - band, 0)
        cb = lo + (rng.random(rb.size) * (np.minimum(rb + band, n - 1) - lo + 1)).astype(np.int64)
        rr = np.repeat(r_all, need_r)
        cr = rng.integers(0, n, rr.size, dtype=np.int64)
        # low bit = draw kind (0 band, 1 uniform): sorting keeps a band draw first
        cand = np.concatenate([(rb * n + cb) << 1, ((rr * n + cr) << 1) | 1])
        cand.sort()
        key = cand >> 1
        first = np.ones(key.size, bool)
        first[1:] = key[1:] != key[:-1]
        if accepted is not None:
            pos = np.searchsorted(accepted, key)
            hit = (pos < accepted.size) & (accepted[np.minimum(pos, accepted.size - 1)] == key)
            if extra.size:
                pe = np.searchsorted(extra, key)
                hit |= (pe < extra.size) & (extra[np.minimum(pe, extra.size - 1)] == key)
            first &= ~hit
        got = key[first]
        kind = (cand[first] & 1).astype(bool)
        rows_got = got // n
        need_b = need_b - np.bincount(rows_got[~kind], minlength=n)
        need_r = need_r - np.bincount(rows_got[kind], minlength=n)
        if accepted is None:
            accepted = got
        else:
            extra = np.sort(np.concatenate([extra, got]))
    else:
        raise RuntimeError("power-law generator did not converge")
    keys = accepted if not extra.size else np.insert(accepted, np.searchsorted(accepted, extra), extra)
    vals = rng.standard_normal(keys.size)
    return _csr_from_sorted_keys(n, keys, vals)


def fem_banded(n: int, rng: np.random.Generator, rl_lo: int = 7, rl_hi: int = 81):
    """One FEM-like banded matrix: row lengths uniform in [rl_lo, rl_hi],
    the diagonal plus rl-1 distinct columns within a band of half-width
    3*rl around it (clipped to [0, n)); off-diagonal values N(0,1), the
    diagonal set to |row sum of the off-diagonals| + 1."""
    rl = rng.integers(rl_lo, rl_hi + 1, n)
    rl = np.minimum(rl, n)
    r_idx = np.arange(n, dtype=np.int64)
    need = rl - 1
    keys = r_idx * n + r_idx  # diagonals
    for _ in range(64):
        if need.sum() == 0:
            break
        rr = np.repeat(r_idx, need)
        w = 3 * rl[rr]
        lo = np.maximum(rr - w, 0)
        hi = np.minimum(rr + w, n - 1)
        cc = lo + (rng.random(rr.size) * (hi - lo + 1)).astype(np.int64)
        allk = np.concatenate([keys, rr * n + cc])
        uk = np.unique(allk)
        cnt = np.bincount(uk // n, minlength=n)
        need = rl - cnt
        keys = uk
        if (need < 0).any():
            raise RuntimeError("fem_banded overfilled a row")
    else:
        raise RuntimeError("fem_banded did not converge")
    row, col, _ = _csr_from_sorted_keys(n, keys, np.zeros(keys.size))
    val = rng.standard_normal(keys.size)
    is_diag = (keys // n) == (keys % n)
    off = np.where(is_diag, 0.0, val)
    rsum = np.add.reduceat(off, row[:-1].astype(np.int64)) if keys.size else np.zeros(n)
    val[is_diag] = np.abs(rsum) + 1.0
    return row, col, val


def fem_batch(count: int = 512, seed: int = 4, n_lo: float = 1e3, n_hi: float = 2e5):
    """`count` FEM-like banded matrices with n log-uniform in [n_lo, n_hi]."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), count)).astype(np.int64)
    return [fem_banded(int(k), rng) for k in ns]


def fem_banded_c(n: int, seed: int, rl_lo: int = 7, rl_hi: int = 81, band: int = 3):
    """The banded FEM-like matrix of fem_banded (same distribution: rl
    uniform in [rl_lo, rl_hi], rl-1 distinct columns uniform within +/-band*rl
    of the diagonal, N(0,1) off-diagonals, diagonal |row sum| + 1) from the
    library's seeded C generator (ispmv_gen_banded: OpenMP over rows,
    SplitMix64 streams per row), fast enough for the full batched workload
    (about 1e9 nonzeros).  Its random stream differs from fem_banded's."""
    import ctypes as C

    from . import abi
    from ._lib import check, load
    lib = load()
    out = abi.StrMatCSR()
    check(lib.ispmv_gen_banded(n, seed, rl_lo, rl_hi, band, C.byref(out)), "ispmv_gen_banded")
    try:
        nnz = out.nnz
        row = np.ctypeslib.as_array(out.row, shape=(n + 1,)).copy()
        col = np.ctypeslib.as_array(out.col, shape=(max(nnz, 1),))[:nnz].copy()
        val = np.ctypeslib.as_array(out.val, shape=(max(nnz, 1),))[:nnz].copy()
    finally:
        lib.ispmv_csr_free(C.byref(out))
    return row, col, val


def fem_batch_c(count: int = 512, seed: int = 4, n_lo: float = 1e3, n_hi: float = 2e5):
    """`count` banded FEM-like matrices with n log-uniform in [n_lo, n_hi]
    (the sizes of fem_batch for the same seed), each from fem_banded_c with
    seed (seed, m)."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), count)).astype(np.int64)
    return [fem_banded_c(int(k), seed * 1_000_003 + m) for m, k in enumerate(ns)]


def uniform_x(n: int, seed: int, k: int | None = None) -> np.ndarray:
    """x ~ U[-1, 1] (FP64), or an n x k row-major block of them."""
    rng = np.random.default_rng(seed)
    if k is None:
        return rng.uniform(-1.0, 1.0, n)
    return rng.uniform(-1.0, 1.0, (n, k))


def random_csr(n: int, seed: int, rl_max: int = 40, empty_frac: float = 0.0, ncols: int | None = None):
    """Small random CSR for tests: row lengths uniform in [0, rl_max] (a
    fraction `empty_frac` forced to 0), distinct sorted columns, N(0,1)."""
    rng = np.random.default_rng(seed)
    ncols = ncols or n
    rl = rng.integers(0, rl_max + 1, n)
    if empty_frac:
        rl[rng.random(n) < empty_frac] = 0
    rl = np.minimum(rl, ncols)
    cols = [np.sort(rng.choice(ncols, int(k), replace=False)) for k in rl]
    row = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(rl, out=row[1:])
    col = np.concatenate(cols).astype(U32) if n else np.zeros(0, U32)
    val = rng.standard_normal(int(row[-1]))
    return row.astype(U32), col, val
