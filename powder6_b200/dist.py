"""Multi-GPU plumbing of the searches: one process per GPU, weak scaling.

Replicas, ladders and searches are independent, so nothing crosses GPUs on
the per-trial path; the collectives are the timing reduction (the maximum
over ranks of each rank's device time) and, at every sync point of a
sharded search, the merge of each rank's per-assignment bests so every rank
holds the global winner of every assignment (the reference keeps one best
per assignment, js/swarm_wyckoff.js:1870-1935), prunes the same assignments
and reports the same result.
The helpers work with the NCCL backend (CUDA tensors) and with gloo (CPU
tensors), which the multi-process tests use.
"""
from __future__ import annotations

import os
from typing import Dict, Tuple

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


def any_over_ranks(flag: bool, world: int) -> bool:
    """True on every rank when any rank's flag is set (a stop request must be
    agreed before the next collective, or the ranks' collectives fall out of
    step)."""
    return bool(max_over_ranks(1.0 if flag else 0.0, world) > 0.5)


def bests_over_ranks(per_assignment: Dict[int, dict], n_assign: int, coords_len: int, scale: float,
                     world: int) -> Dict[int, dict]:
    """The per-assignment best structures of all ranks merged: for every
    assignment the rank whose best has the largest cc - pen x scale (ties to
    the lowest rank) supplies {cc, pen, coords}; every rank gets the same map.
    One all-gather of (score, cc, pen, coords) per assignment per rank; the
    reference keeps exactly one best per assignment (js/swarm_wyckoff.js:1870-1935)."""
    if world == 1:
        return {A: dict(v) for A, v in per_assignment.items()}
    import torch
    import torch.distributed as dist
    dev = _device()
    rec = np.full((n_assign, 3 + coords_len), np.nan, dtype=np.float64)
    rec[:, 0] = -np.inf
    for A, v in per_assignment.items():
        if v.get('coords') is None:
            continue
        rec[A, 0] = float(v['cc']) - float(v['pen']) * scale
        rec[A, 1] = float(v['cc'])
        rec[A, 2] = float(v['pen'])
        rec[A, 3:] = np.asarray(v['coords'], dtype=np.float64).ravel()[:coords_len]
    t = torch.from_numpy(rec).to(dev)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    allr = np.stack([p.cpu().numpy() for p in parts])          # (world, n_assign, 3 + coords)
    out: Dict[int, dict] = {}
    for A in range(n_assign):
        scores = allr[:, A, 0]
        if not np.any(np.isfinite(scores)):
            continue
        r = int(np.argmax(np.where(np.isfinite(scores), scores, -np.inf)))
        row = allr[r, A]
        out[A] = {'cc': float(row[1]), 'pen': float(row[2]), 'coords': row[3:].astype(np.float32), 'rank': r}
    return out


def max_per_assignment(values: Dict[int, float], n_assign: int, world: int) -> Dict[int, float]:
    """Element-wise maximum over ranks of a per-assignment score (absent = -inf)."""
    if world == 1:
        return dict(values)
    import torch
    import torch.distributed as dist
    v = np.full(n_assign, -np.inf, dtype=np.float64)
    for A, x in values.items():
        v[A] = float(x)
    t = torch.from_numpy(v).to(_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    m = t.cpu().numpy()
    return {A: float(m[A]) for A in range(n_assign) if np.isfinite(m[A])}
