"""Voxel-sharded filtered OPW on several GPUs (one process per GPU).

The DAS and the power Doppler are independent per voxel, so every rank
beamforms its own contiguous slab of lateral x planes.  The global SVD clutter
filter needs one exchange: the temporal Gram matrix is a sum over voxel rows
(reference src/rcabeam/gpu_clutter.py:144-160) and its scale is a maximum over
all rows (gpu_clutter.py:141).  Each rank therefore

1. forms its local Casorati scale and all-reduces it with MAX,
2. accumulates its rows' float64 upper-triangle Gram with that global scale
   and all-reduces it (and the row count) with SUM,
3. eigendecomposes the identical T x T matrix redundantly (tiny), projects
   its own rows and keeps its own filtered power;

``gather_power`` assembles the full map where one rank needs it.  Channels are
replicated (each rank receives both apertures).  With NCCL the two all-reduces
move 8 bytes and T^2 x 16 bytes (2.56 MB at T = 400).
"""

from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def x_slab(nx: int, rank: int, world: int) -> slice:
    """Contiguous x-plane range of one rank (sizes differ by at most one plane)."""
    if not 0 <= rank < world or world < 1:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(nx, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def shard_grid(grid, rank: int, world: int):
    """(x, z, y) grid of one rank: its x slab, the full z and y axes."""
    x, z, y = grid
    return (np.asarray(x)[x_slab(len(x), rank, world)], z, y)


def reduce_scale(scale: torch.Tensor, group=None) -> None:
    """Global Casorati scale (max |component| over every rank's rows), in place."""
    if group is not None:
        dist.all_reduce(scale, op=dist.ReduceOp.MAX, group=group)


def reduce_gram(upper: torch.Tensor, rows: int, group=None) -> int:
    """Sum of every rank's upper-triangle Gram partials, in place; returns the total row count."""
    if group is None:
        return rows
    dist.all_reduce(upper, op=dist.ReduceOp.SUM, group=group)
    count = torch.tensor([rows], dtype=torch.int64, device=upper.device)
    dist.all_reduce(count, op=dist.ReduceOp.SUM, group=group)
    return int(count.item())


def gather_power(power: torch.Tensor, group=None) -> torch.Tensor:
    """Concatenate every rank's (nx_local, nz, ny) power along x, in rank order."""
    if group is None:
        return power
    world = dist.get_world_size(group)
    n = torch.tensor([power.shape[0]], dtype=torch.int64, device=power.device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(s.item()) for s in sizes]
    width = max(sizes)
    padded = torch.zeros((width, *power.shape[1:]), dtype=power.dtype, device=power.device)
    padded[: power.shape[0]] = power
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    return torch.cat([p[:s] for p, s in zip(parts, sizes)], dim=0)
