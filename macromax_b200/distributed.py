"""
Multi-GPU use of the solver: replicas only.

A single grid is not sharded (that would need an all-to-all per FFT).  Right-hand sides that share a material are
independent, so N processes (one per GPU) each solve their own contiguous slice of the sources with no data-path
collective; the only collectives are the max-over-ranks of a timing and an optional final gather of the fields.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous slice [start, stop) of n items for ``rank`` of ``world``; sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError('invalid rank/world')
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of a per-rank scalar (e.g. a timing) over all ranks; identity without a process group."""
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_slices(local: torch.Tensor, n_total: int) -> torch.Tensor:
    """Concatenate the per-rank slices [n_local, ...] of ``shard_range`` back into [n_total, ...] on every rank."""
    if not (dist.is_available() and dist.is_initialized()):
        return local
    world = dist.get_world_size()
    sizes = [shard_range(n_total, r, world) for r in range(world)]
    cap = max(b - a for a, b in sizes)
    pad = torch.zeros((cap, *local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[:local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad)
    return torch.cat([p[:b - a] for p, (a, b) in zip(parts, sizes)], dim=0)
