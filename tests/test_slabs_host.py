"""Host logic of the slab decomposition on CPU: row split, neighbours, and the
halo exchange of cfd_inwsl_b200.slabs.exchange_rows over torch.distributed
(gloo, 2 and 3 processes, CPU tensors standing in for device buffers)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cfd_inwsl_b200.slabs import GHOST, exchange_rows, neighbours, slab_rows


def test_slab_rows_cover_the_grid():
    for n, p in [(50, 4), (2048, 8), (36, 3), (17, 3)]:
        rows = slab_rows(n, p)
        assert rows[0][0] == 0 and rows[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(rows, rows[1:]))
        sizes = [r1 - r0 for r0, r1 in rows]
        assert max(sizes) - min(sizes) <= 1


def test_neighbours():
    assert neighbours(0, 4, False) == (None, 1)
    assert neighbours(3, 4, False) == (2, None)
    assert neighbours(0, 4, True) == (3, 1)
    assert neighbours(3, 4, True) == (2, 0)
    assert neighbours(0, 2, True) == (1, 1)
    assert neighbours(0, 1, True) == (0, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def state_of(rank, nvar=4, nrows=7, rowlen=5):
    """A slab state whose every value names (rank, var, row, line)."""
    v, r, l = np.meshgrid(np.arange(nvar), np.arange(nrows), np.arange(rowlen), indexing="ij")
    return torch.tensor(1000.0 * rank + 100.0 * v + 10.0 * r + l / 10.0, dtype=torch.float64)


def _worker(rank, world, port, periodic, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        st = state_of(rank)
        nb = neighbours(rank, world, periodic)
        halo = [torch.full((4, GHOST, 5), np.nan, dtype=torch.float64) if nb[s] is not None else None
                for s in (0, 1)]
        exchange_rows(dist, None, rank, nb, st, halo)
        out[rank] = [h.numpy().copy() if h is not None else None for h in halo]
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,periodic", [(2, True), (2, False), (3, True), (3, False)])
def test_exchange_rows_gloo(world, periodic):
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, periodic, out), nprocs=world, start_method="spawn")
    for rank in range(world):
        lo, hi = neighbours(rank, world, periodic)
        got = out[rank]
        if lo is None:
            assert got[0] is None
        else:  # the low neighbour's last GHOST rows, ascending
            np.testing.assert_array_equal(got[0], state_of(lo).numpy()[:, -GHOST:, :])
        if hi is None:
            assert got[1] is None
        else:  # the high neighbour's first GHOST rows
            np.testing.assert_array_equal(got[1], state_of(hi).numpy()[:, :GHOST, :])


# ------------------------------------------------------------- dt over the ranks
GAMMA = 1.4


def local_words(rank, nrows, rowlen, dim, h):
    """Reduction words of one rank's slab of a random state: [0] a stand-in for
    max |R_rho|, [1..dim] max_cells (c + |u_d|) / h_d as the sweep epilogue
    reduces them (getTimeIntervalExplicit, blockSolver.cpp:318-349)."""
    rng = np.random.default_rng(100 + rank)
    ncell = nrows * rowlen
    rho = rng.uniform(0.1, 2.0, ncell)
    vel = rng.uniform(-1.0, 1.0, (dim, ncell)) * (10.0 ** rng.integers(-3, 2))
    p = rng.uniform(0.05, 2.0, ncell)
    c = np.sqrt(GAMMA * p / rho)
    lam = [np.max((c + np.abs(vel[d])) / h[d]) for d in range(dim)]
    words = [rng.uniform(0, 1) * 10.0 ** rng.integers(-300, 300)] + lam + [0.0] * (3 - dim)
    return np.array(words), (rho, vel, p)


def _dt_worker(rank, world, port, dim, out):
    from cfd_inwsl_b200.slabs import allreduce_max_words, dt_from_words, words_from_wave_speeds
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        h = [0.01, 0.02, 0.005][:dim]
        vals, _ = local_words(rank, 6, 9, dim, h)
        words = torch.from_numpy(words_from_wave_speeds(vals))
        allreduce_max_words(dist, None, words)
        out[rank] = (words.numpy().copy(), dt_from_words(words.numpy(), dim, 0.5))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,dim", [(2, 2), (3, 3), (3, 2)])
def test_dt_from_max_allreduce_of_words_gloo(world, dim):
    """The per-step MAX all-reduce of the int64 reduction words gives every
    rank the global maxima bit for bit, and the dt built from them equals the
    reference formula CFL / sum_d max (c + |u_d|) / h_d over the undivided grid."""
    from cfd_inwsl_b200.slabs import wave_speeds_from_words
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_dt_worker, args=(world, port, dim, out), nprocs=world, start_method="spawn")
    h = [0.01, 0.02, 0.005][:dim]
    per_rank = [local_words(r, 6, 9, dim, h) for r in range(world)]
    want = np.max([w for w, _ in per_rank], axis=0)
    # the undivided grid: every rank's cells together
    rho = np.concatenate([s[0] for _, s in per_rank])
    vel = np.concatenate([s[1] for _, s in per_rank], axis=1)
    p = np.concatenate([s[2] for _, s in per_rank])
    c = np.sqrt(GAMMA * p / rho)
    lam_total = 0.0
    for d in range(dim):
        lam_total += np.max((c + np.abs(vel[d])) / h[d])
    dt_whole = 0.5 / lam_total
    for r in range(world):
        words, dt = out[r]
        np.testing.assert_array_equal(wave_speeds_from_words(words), want)
        assert dt == dt_whole


def test_words_order_like_the_doubles():
    """IEEE bit patterns of non-negative doubles order like the doubles,
    subnormals, zero and huge values included; negative or NaN inputs are refused."""
    from cfd_inwsl_b200.slabs import wave_speeds_from_words, words_from_wave_speeds
    vals = np.array([0.0, 5e-324, 2.2e-308, 1e-300, 0.5, 1.0, 1.0000000000000002, 3e10, 1e308, np.inf])
    w = words_from_wave_speeds(vals)
    assert np.all(np.diff(w) > 0)
    np.testing.assert_array_equal(wave_speeds_from_words(w), vals)
    rng = np.random.default_rng(5)
    a, b = rng.uniform(0, 1e6, 1000), rng.uniform(0, 1e6, 1000)
    np.testing.assert_array_equal(wave_speeds_from_words(np.maximum(words_from_wave_speeds(a),
                                                                    words_from_wave_speeds(b))), np.maximum(a, b))
    with pytest.raises(ValueError):
        words_from_wave_speeds([-1.0])
    with pytest.raises(ValueError):
        words_from_wave_speeds([np.nan])
