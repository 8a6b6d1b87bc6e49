"""Multi-GPU plumbing: one process per GPU, cells sharded by contiguous ranges.

Cells are independent, so a multi-GPU solve needs no exchange while it
integrates: each rank solves its own contiguous range of cells (aligned to
the lockstep group size so no group straddles two ranks) and, if the caller
wants the whole state on every rank, the ranges are gathered once at the end.
Timings are reduced with MAX over ranks.  torch.distributed provides the
process group (NCCL on GPUs, gloo on CPUs).
"""
from __future__ import annotations

from typing import Tuple

import numpy as np


def cell_range(ncells: int, rank: int, world: int, align: int = 1) -> Tuple[int, int]:
    """[start, stop) of this rank's cells: contiguous, sizes differing by at
    most `align`, every boundary a multiple of `align`."""
    if ncells % align:
        raise ValueError("ncells %d is not a multiple of the group size %d" % (ncells, align))
    groups = ncells // align
    base, extra = divmod(groups, world)
    g0 = rank * base + min(rank, extra)
    g1 = g0 + base + (1 if rank < extra else 0)
    return g0 * align, g1 * align


def max_over_ranks(value: float) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_cells(local: np.ndarray, ncells: int, align: int = 1) -> np.ndarray:
    """All ranks' cell ranges of a (..., local_cells) array, reassembled to
    (..., ncells) on every rank (one all_gather at the end of a solve)."""
    import torch
    import torch.distributed as dist
    world, rank = dist.get_world_size(), dist.get_rank()
    sizes = [cell_range(ncells, r, world, align) for r in range(world)]
    width = max(b - a for a, b in sizes)
    lead = local.shape[:-1]
    pad = np.zeros(lead + (width,), dtype=local.dtype)
    pad[..., : local.shape[-1]] = local
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else "cpu"
    t = torch.from_numpy(pad).to(dev)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    out = np.empty(lead + (ncells,), dtype=local.dtype)
    for r, (a, b) in enumerate(sizes):
        out[..., a:b] = parts[r].cpu().numpy()[..., : b - a]
    return out
