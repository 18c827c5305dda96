"""Replica sharding across ranks (host logic of the multi-GPU path), on CPU: the split covers every replica once
and balances site counts; two gloo ranks agree on it without communicating, gather each other's per-replica
results and take the maximum of their timings."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from mclics_b200 import sharding


def c3_sizes():
    import numpy as np
    rng = np.random.default_rng(11)
    L = 2 * np.round(np.exp(rng.uniform(np.log(16), np.log(128), 64)) / 2).astype(int)
    return [int(l) ** 3 for l in L]


def test_partition_covers_and_balances():
    sizes = c3_sizes()
    for world in (1, 2, 3, 4, 8):
        parts = sharding.partition(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in p) for p in parts]
        # greedy largest-first: the spread is at most the largest replica
        assert max(loads) - min(loads) <= max(sizes)
    assert sharding.partition([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]
    assert sharding.partition([], 3) == [[], [], []]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        sizes = c3_sizes()
        mine = sharding.shard(sizes, world, rank)
        local = {i: {"rank": rank, "sites": sizes[i]} for i in mine}
        merged = sharding.gather_results(local, world)
        slowest = sharding.max_over_ranks(1.0 + rank, world)
        q.put((rank, sorted(merged), [merged[i]["rank"] for i in sorted(merged)], slowest))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_the_batch():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = sharding.partition(c3_sizes(), world)
    for rank, keys, owners, slowest in got:
        assert keys == list(range(64))
        assert all(i in parts[o] for i, o in zip(keys, owners))
        assert slowest == 2.0
