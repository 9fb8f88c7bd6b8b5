"""Multi-GPU sharding of independent grids: the host logic on CPU.

The batched workload splits whole grids across ranks (greedy LPT on a
per-grid cost estimate) with no collective on the data path; only the
reported totals are reduced.  These tests run without a GPU: the partition's
properties directly, and the rank protocol as two gloo processes.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from sharc.volrus_b200.method import random_sphere_grids
from sharc.volrus_b200.shard import imbalance, partition_lpt, reduce_totals, shard_of, sphere_grid_cost


def test_partition_covers_every_item_once_and_is_deterministic():
    rng = np.random.default_rng(5)
    costs = rng.lognormal(3.0, 1.5, 257)
    for world in (1, 2, 3, 4, 8):
        parts = partition_lpt(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        assert parts == partition_lpt(costs, world)
        assert all(p == sorted(p) for p in parts)


def test_partition_balances_the_batched_workload():
    grids = random_sphere_grids(256, seed=3)
    costs = [sphere_grid_cost(g[0]) for g in grids]
    for world in (2, 4, 8):
        assert imbalance(costs, partition_lpt(costs, world)) < 1.05


def test_partition_edge_cases():
    assert partition_lpt([], 4) == [[], [], [], []]
    assert partition_lpt([5.0], 3) == [[0], [], []]
    assert partition_lpt([1.0, 1.0, 1.0, 1.0], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        partition_lpt([1.0], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        grids = random_sphere_grids(40, seed=9)
        mine, idx = shard_of(grids, rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, idx)
        local = float(sum(sphere_grid_cost(g[0]) for g in mine))
        total, tmax = reduce_totals(local, 1.0 + rank)
        q.put((rank, gathered, local, total, tmax))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_disjointly_and_reduce_totals():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    grids = random_sphere_grids(40, seed=9)
    costs = [sphere_grid_cost(g[0]) for g in grids]
    gathered = out[0][1]
    assert gathered == out[1][1]
    assert sorted(i for part in gathered for i in part) == list(range(40))
    assert not set(gathered[0]) & set(gathered[1])
    want_total = float(sum(costs))
    for rank, _, local, total, tmax in out:
        assert abs(total - want_total) <= 1e-9 * want_total
        assert tmax == 2.0
    assert abs(out[0][2] + out[1][2] - want_total) <= 1e-9 * want_total


def test_reduce_totals_without_process_group():
    assert reduce_totals(12.5, 3.0) == (12.5, 3.0)
