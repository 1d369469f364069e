"""Synthetic workload generators (sizes and distributions the benchmark
configurations state) and the multi-process timing reduction bench.py uses
(max over ranks), run as world-size-2 gloo ranks on the CPU."""
from __future__ import annotations

import os

import numpy as np
import pytest

from int_spmv_b200 import matrices as M


def test_poisson_sizes():
    row, col, val = M.poisson2d(512)
    n = 512 * 512
    assert len(row) - 1 == n and len(col) == 5 * n - 4 * 512 == 1308672
    assert np.all(val[row[:-1][:3] + 0] <= 4.0)
    rl = np.diff(row.astype(np.int64))
    assert rl.min() == 3 and rl.max() == 5
    k = np.repeat(np.arange(n, dtype=np.int64), rl) * n + col
    assert np.all(np.diff(k) > 0)


def test_stencil27_small():
    m = 12
    row, col, val = M.stencil27(m, seed=2)
    n = m ** 3
    assert len(col) == (3 * m - 2) ** 3
    rl = np.diff(row.astype(np.int64))
    assert rl.min() == 8 and rl.max() == 27
    r = np.repeat(np.arange(n), rl)
    diag = r == col
    assert np.all(val[diag] == 26.0)
    assert np.all((val[~diag] >= -1.1) & (val[~diag] <= -0.9))
    assert np.array_equal(M.stencil27(m, seed=2)[2], val)  # seeded


def test_powerlaw_properties():
    n = 200_000
    row, col, val = M.powerlaw(n, seed=1)
    rl = np.diff(row.astype(np.int64))
    assert rl.min() >= 1 and rl.max() <= 5000
    assert 13.5 < rl.mean() < 16.5  # lognormal(2.2, 1): mean e^2.7 = 14.9
    r = np.repeat(np.arange(n, dtype=np.int64), rl)
    k = r * n + col
    assert np.all(np.diff(k) > 0)  # distinct, sorted in each row
    band = np.abs(r - col.astype(np.int64)) <= 1000
    assert 0.69 < band.mean() < 0.72
    assert abs(val.mean()) < 0.01 and abs(val.std() - 1) < 0.01
    row2, col2, val2 = M.powerlaw(n, seed=1)
    assert np.array_equal(col, col2) and np.array_equal(val, val2)


def test_fem_batch_small():
    mats = M.fem_batch(count=6, seed=4, n_lo=1000, n_hi=3000)
    assert len(mats) == 6
    for row, col, val in mats:
        n = len(row) - 1
        rl = np.diff(row.astype(np.int64))
        assert rl.min() >= 7 and rl.max() <= 81
        r = np.repeat(np.arange(n), rl)
        assert np.all(np.abs(r - col.astype(np.int64)) <= 3 * 81)
        d = val[r == col]
        off = np.abs(np.where(r == col, 0, val))
        assert np.all(d >= 1.0)


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    v = bench.max_over_ranks(1.0 + rank * 2.5, world, device="cpu")
    bench.barrier(world)
    q.put((rank, v))
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import multiprocessing as mp
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    assert res == {0: 3.5, 1: 3.5}


def test_gen_banded_invariants():
    """The C generator of the batched workload: row lengths, band, distinct
    ascending columns with the diagonal, diagonal = |off-diagonal sum| + 1,
    N(0,1) off-diagonals, and determinism."""
    from int_spmv_b200 import matrices as M
    for n, seed in ((1, 3), (9, 4), (1000, 5), (20011, 6)):
        row, col, val = M.fem_banded_c(n, seed)
        rl = np.diff(row.astype(np.int64))
        assert np.all(rl >= min(7, n)) and np.all(rl <= min(81, n))
        rows = np.repeat(np.arange(n), rl)
        assert np.all(np.abs(col.astype(np.int64) - rows) <= 3 * rl[rows])
        # ascending, distinct within each row
        d = np.diff(col.astype(np.int64))
        inner = np.ones(len(col), bool)
        inner[row[1:-1].astype(np.int64)] = False
        assert np.all(d[inner[1:]] > 0)
        diag = col.astype(np.int64) == rows
        assert np.array_equal(np.bincount(rows[diag], minlength=n), np.ones(n, np.int64))
        offsum = np.bincount(rows[~diag], weights=val[~diag], minlength=n)
        assert np.allclose(val[diag], np.abs(offsum) + 1.0)
        r2, c2, v2 = M.fem_banded_c(n, seed)
        assert np.array_equal(row, r2) and np.array_equal(col, c2) and np.array_equal(val, v2)
    off = val[~diag]
    assert abs(off.mean()) < 0.01 and abs(off.std() - 1.0) < 0.01
    # uniform within the band: the mean offset is near 0 and |offset|/(3*rl) near 1/2
    offs = (col.astype(np.int64) - rows)[~diag] / (3.0 * rl[rows][~diag])
    interior = (rows[~diag] > 300) & (rows[~diag] < n - 300)
    assert abs(offs[interior].mean()) < 0.01 and abs(np.abs(offs[interior]).mean() - 0.5) < 0.01


def test_fem_batch_c_sizes_match_fem_batch():
    from int_spmv_b200 import matrices as M
    mats = M.fem_batch_c(count=6, seed=4, n_lo=1e3, n_hi=3e3)
    rng = np.random.default_rng(4)
    ns = np.exp(rng.uniform(np.log(1e3), np.log(3e3), 6)).astype(np.int64)
    assert [len(r) - 1 for r, _, _ in mats] == list(ns)
