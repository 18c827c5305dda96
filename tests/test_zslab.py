"""Host logic of the z-slab decomposition, on CPU: the plane partition and neighbour map, and the boundary-plane
exchange and the sums' all-reduce through torch.distributed with gloo ranks (2 and 3 ranks, periodic and free z).
Every rank fills its send buffers with values that name the rank and the side; after one exchange each receive
buffer must hold exactly the neighbour's plane that the decomposition puts there (lower halo = the lower
neighbour's highest owned plane, upper halo = the upper neighbour's lowest)."""
import datetime
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

from mclics_b200 import zslab


def test_partition_and_neighbours():
    assert zslab.partition(30, 3) == [(0, 10), (10, 10), (20, 10)]
    assert zslab.partition(31, 4) == [(0, 8), (8, 8), (16, 8), (24, 7)]
    for nz in (1, 7, 256):
        for world in range(1, min(nz, 9) + 1):
            parts = zslab.partition(nz, world)
            assert sum(n for _, n in parts) == nz
            assert all(parts[i][0] + parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            assert max(n for _, n in parts) - min(n for _, n in parts) <= 1
    with pytest.raises(ValueError):
        zslab.partition(3, 4)
    assert zslab.neighbours(0, 3, True) == (2, 1)
    assert zslab.neighbours(2, 3, True) == (1, 0)
    assert zslab.neighbours(0, 3, False) == (None, 1)
    assert zslab.neighbours(2, 3, False) == (1, None)
    assert zslab.neighbours(0, 1, True) == (0, 0)
    assert zslab.neighbours(0, 1, False) == (None, None)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _plane(rank, side, n=37):
    # a plane that names its rank and side: side 0 = lowest owned plane, 1 = highest
    return torch.arange(n, dtype=torch.float32) + 1000.0 * rank + 100.0 * side


def _rank(rank, world, periodic, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ex = zslab.TorchExchange()
        lo, hi = zslab.neighbours(rank, world, periodic)
        send_lo, send_hi = _plane(rank, 0), _plane(rank, 1)
        recv_lo, recv_hi = torch.full_like(send_lo, -1.0), torch.full_like(send_hi, -1.0)
        ex.exchange(rank, lo, hi, send_lo, send_hi, recv_lo, recv_hi)
        sums = torch.arange(zslab.N_SUMS, dtype=torch.float64) * (rank + 1)
        ex.allreduce(sums)
        q.put((rank, lo, hi, recv_lo.tolist(), recv_hi.tolist(), sums.tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,periodic", [(2, True), (2, False), (3, True), (3, False)])
def test_exchange_and_allreduce_over_gloo(world, periodic):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, periodic, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    tri = world * (world + 1) / 2
    for rank, lo, hi, recv_lo, recv_hi, sums in got:
        if lo is None:
            assert recv_lo == [-1.0] * len(recv_lo)
        else:
            assert recv_lo == _plane(lo, 1).tolist()  # the lower neighbour's highest owned plane
        if hi is None:
            assert recv_hi == [-1.0] * len(recv_hi)
        else:
            assert recv_hi == _plane(hi, 0).tolist()  # the upper neighbour's lowest owned plane
        assert sums == [k * tri for k in range(zslab.N_SUMS)]


def test_single_periodic_rank_wraps_onto_itself():
    ex = zslab.TorchExchange()
    send_lo, send_hi = _plane(0, 0), _plane(0, 1)
    recv_lo, recv_hi = torch.zeros_like(send_lo), torch.zeros_like(send_hi)
    ex.exchange(0, 0, 0, send_lo, send_hi, recv_lo, recv_hi)  # no process group needed
    assert torch.equal(recv_lo, send_hi) and torch.equal(recv_hi, send_lo)
