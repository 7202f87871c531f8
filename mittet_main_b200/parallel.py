"""Multi-GPU plumbing: shots are independent (the reference's source-position
loop, ncver0027/cpu_main.f90:35, satan_i/fwi3d_cpu_rec2rec_v1.4.c:38), so
each rank (one process per GPU) holds a replica of the model and solves its
own shots; the only collective is the sum of the per-rank FWI gradients
(and misfits), one all-reduce of nx*ny*nz doubles per gradient evaluation.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def shard_shots(nshot: int, rank: int, world: int) -> list[int]:
    """Contiguous, balanced block of shot indices for one rank."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(nshot, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


def distributed_gradient(local_gradient: Callable[[Sequence[int]], tuple[float, np.ndarray]], nshot: int,
                         group=None) -> tuple[float, np.ndarray]:
    """Sum over all shots of (misfit, gradient), each rank computing its shard.

    local_gradient(shot_indices) -> (misfit, grad) for those shots on this rank
    (an empty shard returns (0, zeros)).  Uses torch.distributed (NCCL across
    GPUs, gloo on the CPU); every rank receives the total."""
    import torch
    import torch.distributed as dist

    rank = dist.get_rank(group) if dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    mine = shard_shots(nshot, rank, world)
    mis, grad = local_gradient(mine)
    if world == 1:
        return mis, grad
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.from_numpy(np.concatenate([[mis], grad.ravel()])).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    out = t.cpu().numpy()
    return float(out[0]), out[1:].reshape(grad.shape)
