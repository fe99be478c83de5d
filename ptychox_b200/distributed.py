"""Data-parallel sweeps: one process per GPU, positions sharded, one gradient exchange.

A sweep's units (scan positions, LEDs, diversity shifts) are independent; the only
exchange step is the sum of the per-rank gradients (and losses).  Each rank sweeps its
shard with the fused kernels and then calls :func:`reduce_sweep`, which turns the rank's
mean loss and its gradients into those of the global mean over all units with one
all-reduce per tensor (NCCL over NVLink/NVSwitch on GPUs, gloo in the CPU tests).

Shards are contiguous bands of object rows (positions sorted by y, then x), so each
rank's object-gradient scatter stays inside its band.
"""

from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

__all__ = ["shard_positions", "reduce_sweep"]


def shard_positions(positions_xy, rank: int, world: int) -> np.ndarray:
    """Indices of the units of ``rank``: contiguous row bands, sizes differing by at most one."""
    pos = np.asarray(positions_xy.cpu() if isinstance(positions_xy, torch.Tensor) else positions_xy)
    if not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    order = np.lexsort((pos[:, 0], pos[:, 1])) if pos.ndim == 2 and pos.shape[1] == 2 else np.arange(len(pos))
    bounds = np.linspace(0, len(order), world + 1).round().astype(np.int64)
    return np.sort(order[bounds[rank]:bounds[rank + 1]])


def reduce_sweep(loss: torch.Tensor, grads: list[torch.Tensor], local_units: int, total_units: int,
                 group=None) -> None:
    """In place: ``loss`` and ``grads`` of this rank's mean -> those of the global mean.

    Rank r's loss is the mean over its ``local_units`` units, so the global mean is
    ``sum_r (local_r / total) loss_r`` and likewise for every gradient.
    """
    w = float(local_units) / float(total_units)
    for t in [loss, *grads]:
        t.mul_(w)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
