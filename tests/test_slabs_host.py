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
