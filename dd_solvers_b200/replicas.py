"""Multi-GPU replicas: right-hand sides split over ranks, no exchange in the solve.

The reference is single-GPU; the measured workloads need no data exchange
between GPUs, so ``bench.py --gpus N`` runs one process per GPU (torchrun),
each solving its own right-hand sides on its own copy of the problem. These
helpers are the only cross-rank logic: the RHS split, the per-rank seeds,
and the max-over-ranks reduction of device times (any backend: NCCL on GPUs,
gloo in the CPU tests).
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def rhs_range(total: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous share of ``total`` right-hand sides for ``rank`` (sizes differ by at most one)."""
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def rhs_seed(rank: int, step: int) -> int:
    """Seed of the right-hand side solved by ``rank`` at ``step`` (distinct across ranks)."""
    return 1000 * rank + step


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar (e.g. a CUDA-event time) over the process group."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t)


def gather_columns(local: torch.Tensor, total: int) -> torch.Tensor:
    """All-gather the (n, R_rank) solution blocks of every rank into (n, total)."""
    world = dist.get_world_size()
    width = -(-total // world)  # shares padded to equal width (collectives need equal sizes)
    padded = torch.zeros(local.shape[0], width, dtype=local.dtype, device=local.device)
    padded[:, :local.shape[1]] = local
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded)
    cols = []
    for r in range(world):
        a, b = rhs_range(total, r, world)
        cols.append(parts[r][:, :b - a])
    return torch.cat(cols, dim=1)
