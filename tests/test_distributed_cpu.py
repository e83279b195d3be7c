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


def _columns_worker(rank, world, port, q):
    """Each rank of a 2-rank gloo group computes its shard of the scattering-matrix columns; the per-rank solve is
    replaced by a host function of the mode vectors, so the partition and the gather are what is tested."""
    import numpy as np
    import torch.distributed as dist
    from macromax_b200 import Grid
    from macromax_b200.matrix import ScatteringMatrix
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        grid = Grid(shape=(32, 16), step=0.125)
        sm = ScatteringMatrix(grid, vectorial=True, vacuum_wavelength=0.5, epsilon=1.0, dtype=np.complex128)
        seen = []

        def local(vectors):
            seen.append(vectors.shape[0])
            flat = vectors.reshape(vectors.shape[0], -1)
            return (flat * (2.0 + 1.0j) + np.arange(flat.shape[1])).astype(np.complex128)

        sm._outward_local = local
        rng = np.random.default_rng(0)
        B = 7
        vec = rng.standard_normal((B, 2, 2, sm._modes.size)) + 1j * rng.standard_normal((B, 2, 2, sm._modes.size))
        out = sm._batched_outward(vec)
        q.put((rank, seen, np.allclose(out, local(vec)), out.shape))
    finally:
        dist.destroy_process_group()


def test_scattering_matrix_columns_shard_over_two_gloo_ranks():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = 29600 + os.getpid() % 1000
    procs = [ctx.Process(target=_columns_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    results = sorted(q.get(timeout=10) for _ in range(2))
    # rank 0 solves columns 0..3, rank 1 columns 4..6; both end with all 7, equal to the unsharded result
    assert [r[1][0] for r in results] == [4, 3]
    for rank, seen, equal, shape in results:
        assert equal and shape[0] == 7


class _FakeBatch:
    """Stands in for BatchSolution in the sharding tests: the 'solution' of source k is a fixed function of it."""
    seen = []

    def __init__(self, grid, sources, epsilon, **kwargs):
        import numpy as np
        self.src = np.asarray(sources)
        _FakeBatch.seen.append(int(self.src.shape[0]))

    def solve(self, rtol, maxiter):
        return self

    @property
    def E(self):
        return (self.src * (2.0 + 1.0j)).astype('complex64')

    @property
    def iterations(self):
        return self.src[:, 0, 0, 0].real.astype('int32')

    @property
    def residues(self):
        return self.src[:, 0, 0, 0].real * 0.5

    def close(self):
        pass


def _sources(n=7):
    import numpy as np
    src = np.random.default_rng(5).standard_normal((n, 1, 6, 4)).astype(np.complex64)
    src[:, 0, 0, 0] = np.arange(n)
    return src


def _batch_worker(rank, world, port, q):
    import numpy as np
    import torch.distributed as dist
    from macromax_b200 import Grid, batch
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        batch.BatchSolution = _FakeBatch
        src = _sources()
        out = batch.solve_sharded(Grid(shape=(6, 4), step=0.125), src, 1.0, vacuum_wavelength=0.5)
        ok = (np.array_equal(out['E'], (src * (2.0 + 1.0j)).astype(np.complex64))
              and out['iterations'].tolist() == list(range(7)) and np.allclose(out['residues'], np.arange(7) * 0.5))
        q.put((rank, list(_FakeBatch.seen), bool(ok), out['E'].shape))
    finally:
        dist.destroy_process_group()


def test_batch_sources_shard_over_two_gloo_ranks():
    """solve_sharded: each of two gloo ranks solves its shard_range slice of 7 sources (4 and 3) and both end with all
    7 fields, iteration counts and residues in source order."""
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = 29700 + os.getpid() % 1000
    procs = [ctx.Process(target=_batch_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    results = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in results] == [[4], [3]]
    for rank, seen, ok, shape in results:
        assert ok and shape == (7, 1, 6, 4)


def test_batch_sources_without_a_process_group_solve_all(monkeypatch):
    import numpy as np
    from macromax_b200 import Grid, batch
    monkeypatch.setattr(batch, 'BatchSolution', _FakeBatch)
    _FakeBatch.seen = []
    src = _sources(5)
    out = batch.solve_sharded(Grid(shape=(6, 4), step=0.125), src, 1.0, vacuum_wavelength=0.5)
    assert _FakeBatch.seen == [5]
    assert np.array_equal(out['E'], (src * (2.0 + 1.0j)).astype(np.complex64))
    assert out['iterations'].tolist() == list(range(5))
