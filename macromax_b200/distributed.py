"""
Multi-GPU use of the solver: replicas only.

A single grid is not sharded (that would need an all-to-all per FFT).  Right-hand sides that share a material are
independent, so N processes (one per GPU) each solve their own contiguous slice of the sources with no data-path
collective; the only collectives are the max-over-ranks of a timing and the final gather of the results
(``ScatteringMatrix`` gathers its columns' detection vectors this way under ``torchrun``, and
``batch.solve_sharded`` the fields of a batch of sources).
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


def world() -> tuple[int, int]:
    """(rank, world size) of the default process group, (0, 1) without one."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def gather_rows(local, n_total: int):
    """``gather_slices`` for host arrays (numpy, real or complex): every rank's ``shard_range`` slice of the rows,
    concatenated in rank order on every rank.  The rows travel as a tensor on the device the process group's backend
    needs (CUDA for NCCL, the host for gloo)."""
    import numpy as np
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return local
    local = np.ascontiguousarray(local)
    t = torch.from_numpy(local)
    if t.is_complex():
        t = torch.view_as_real(t)
    if dist.get_backend() == 'nccl':
        t = t.cuda()
    full = gather_slices(t, n_total).cpu()
    if np.iscomplexobj(local):
        full = torch.view_as_complex(full.contiguous())
    return full.numpy().astype(local.dtype, copy=False)
