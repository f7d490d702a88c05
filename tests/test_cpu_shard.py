"""Multi-rank host logic on CPU (gloo, world size 2): the zig-zag frequency
ownership covers every frequency exactly once and balances the work, and
the max-over-ranks step time is what the benchmark reports."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from dsmsgt.shard import owned_freqs, owns


def test_zigzag_partition_single_process():
    for nproc in (1, 2, 3, 4, 8):
        imax = 257
        seen = []
        for p in range(nproc):
            seen += owned_freqs(0, imax, p, nproc)
        assert sorted(seen) == list(range(1, imax + 1))
        # cost ~ frequency (cutoff grows with omega): balanced within one pair
        costs = [sum(owned_freqs(0, imax, p, nproc)) for p in range(nproc)]
        assert max(costs) - min(costs) <= 2 * imax
    assert not owns(0, 100, 0, 1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, imax, out):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    mine = owned_freqs(0, imax, rank, world)
    lists = [None] * world
    dist.all_gather_object(lists, mine)
    t = torch.tensor([0.5 + rank], dtype=torch.float64)  # a per-rank step time
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        out.put((lists, float(t.item())))
    dist.barrier()
    dist.destroy_process_group()


def test_zigzag_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    imax = 64
    procs = [ctx.Process(target=_worker, args=(r, 2, port, imax, q)) for r in range(2)]
    for p in procs:
        p.start()
    lists, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    a, b = lists
    assert not set(a) & set(b)
    assert sorted(a + b) == list(range(1, imax + 1))
    assert tmax == pytest.approx(1.5)
