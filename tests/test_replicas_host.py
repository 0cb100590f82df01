"""Replica sharding of independent cases (cfd_inwsl_b200.replicas) on CPU:
the cost partition, and run_sharded's gather over torch.distributed with gloo
(2 and 3 processes; a stand-in for the per-rank batch run)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from cfd_inwsl_b200 import cases
from cfd_inwsl_b200.replicas import case_cost, partition_by_cost, run_sharded, share_loads


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_partition_of_the_batched_configuration(world):
    """The 256 cases of the batched configuration (N = 129..1018): every case
    once, ascending lists, the same partition on every call, and the largest
    share within the longest-processing-time bound of 4/3 of the lower bound
    max(total / world, largest case)."""
    sizes, _ = cases.riemann_batch(256, 0)
    costs = [case_cost(n) for n in sizes]
    shares = partition_by_cost(costs, world)
    assert partition_by_cost(costs, world) == shares
    flat = sorted(i for s in shares for i in s)
    assert flat == list(range(len(sizes)))
    assert all(s == sorted(s) for s in shares)
    loads = share_loads(costs, shares)
    lower = max(sum(costs) / world, max(costs))
    assert max(loads) <= 4.0 / 3.0 * lower
    if world > 1:
        assert max(loads) / min(loads) < 1.05, loads  # many small cases: nearly even


def test_partition_edge_cases():
    assert partition_by_cost([], 3) == [[], [], []]
    assert partition_by_cost([5.0], 3) == [[0], [], []]
    assert partition_by_cost([1.0, 1.0, 1.0, 1.0], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        partition_by_cost([1.0], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, costs, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        items = list(range(len(costs)))
        # each "case" returns its index squared and the rank that ran it
        res = run_sharded(items, lambda idx: [(i * i, rank) for i in idx], costs, rank, world)
        out[rank] = res
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_run_sharded_gathers_in_order(world):
    rng = np.random.default_rng(world)
    costs = [case_cost(int(n)) for n in rng.integers(16, 200, size=23)]
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(world, _free_port(), costs, out), nprocs=world, join=True)
    assert out[1] is None
    res = out[0]
    assert [v for v, _ in res] == [i * i for i in range(len(costs))]
    shares = partition_by_cost(costs, world)
    for r, s in enumerate(shares):
        assert all(res[i][1] == r for i in s)
