"""Replicas across GPUs: independent lattices need no exchange, so a batch is split across ranks by site count
(greedy, largest first onto the least loaded rank) and every rank sweeps its share with no data-path collective.
The only collectives are host-side: gathering the per-replica results and the slowest rank's time.

    mine = shard(sizes, world, rank)        # indices of this rank's replicas
"""


def partition(sizes, world):
    """Replica indices per rank: each replica, largest first, goes to the rank with the fewest sites so far
    (ties: the lower rank). Deterministic, so every rank computes the same split without communication."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


def shard(sizes, world, rank):
    return partition(sizes, world)[rank]


def gather_results(local, world, group=None):
    """All ranks' {replica index: result} dicts merged on every rank (torch.distributed object all-gather)."""
    import torch.distributed as dist
    if world == 1:
        return dict(local)
    out = [None] * world
    dist.all_gather_object(out, dict(local), group=group)
    merged = {}
    for d in out:
        merged.update(d)
    return merged


def max_over_ranks(value, world, group=None):
    """The largest of the ranks' values (e.g. device seconds), on every rank."""
    import torch
    import torch.distributed as dist
    if world == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t[0])
