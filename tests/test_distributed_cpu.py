"""Replica sharding helpers on two gloo ranks (CPU): slices cover every right-hand side once; max-over-ranks."""
import os

import pytest
import torch
import torch.multiprocessing as mp

from macromax_b200.distributed import shard_range


def test_shard_range_partitions():
    for n in (0, 1, 5, 256):
        for world in (1, 2, 3, 8):
            parts = [shard_range(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from macromax_b200.distributed import gather_slices, max_over_ranks, shard_range
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        n = 7
        a, b = shard_range(n, rank, world)
        local = torch.arange(a, b, dtype=torch.float64).reshape(-1, 1) * torch.ones(1, 3, dtype=torch.float64)
        full = gather_slices(local, n)
        t = max_over_ranks(1.0 + rank)
        q.put((rank, full[:, 0].tolist(), t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_and_max():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    results = sorted(q.get(timeout=10) for _ in range(2))
    for rank, full, t in results:
        assert full == [0.0, 1.0, 2.0, 3.0, 4.0, 5.0, 6.0]
        assert t == 2.0
