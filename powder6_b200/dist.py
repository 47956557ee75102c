"""Multi-GPU plumbing of the searches: one process per GPU, weak scaling.

Replicas, ladders and searches are independent, so nothing crosses GPUs on
the per-trial path; the collectives are the timing reduction (the maximum
over ranks of each rank's device time) and, at a sync point, the exchange
of each rank's best structure so every rank reports the global winner (the
reference keeps one best per assignment, js/swarm_wyckoff.js:1870-1935).
The helpers work with the NCCL backend (CUDA tensors) and with gloo (CPU
tensors), which the multi-process tests use.
"""
from __future__ import annotations

import os
from typing import Tuple

import numpy as np


def world_rank() -> Tuple[int, int, int]:
    return (int(os.environ.get('WORLD_SIZE', '1')), int(os.environ.get('RANK', '0')),
            int(os.environ.get('LOCAL_RANK', '0')))


def _device():
    import torch
    import torch.distributed as dist
    return torch.device('cuda') if dist.get_backend() == 'nccl' else torch.device('cpu')


def max_over_ranks(x: float, world: int) -> float:
    """The largest of every rank's x (the job's time is its slowest rank's)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def best_over_ranks(score: float, coords: np.ndarray, world: int) -> Tuple[float, np.ndarray, int]:
    """Max-loc of (score, coords) over ranks: every rank gets the winner's
    score, coordinates and rank (ties go to the lowest rank)."""
    coords = np.asarray(coords, dtype=np.float32).ravel()
    if world == 1:
        return float(score), coords.copy(), 0
    import torch
    import torch.distributed as dist
    dev = _device()
    s = torch.tensor([float(score)], dtype=torch.float64, device=dev)
    scores = [torch.zeros_like(s) for _ in range(world)]
    dist.all_gather(scores, s)
    vals = [float(v.item()) for v in scores]
    win = int(np.argmax(vals))
    c = torch.from_numpy(coords.copy()).to(dev)
    dist.broadcast(c, src=win)
    return vals[win], c.cpu().numpy(), win


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
