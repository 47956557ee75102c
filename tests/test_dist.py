"""Multi-rank host logic on CPU: two gloo ranks (the path bench.py takes
under torchrun with NCCL, one process per GPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from powder6_b200.dist import barrier, best_over_ranks, max_over_ranks, sum_over_ranks, world_rank
        w, r, lr = world_rank()
        t = max_over_ranks(10.0 + r, w)
        n = sum_over_ranks(1000 * (r + 1), w)
        coords = np.full(6, float(r), dtype=np.float32)
        best, c, win = best_over_ranks(0.5 + 0.1 * r, coords, w)
        barrier(w)
        q.put((rank, w, r, t, n, best, c.tolist(), win))
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_sum_and_best():
    world = 2
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, w, r, t, n, best, c, win in out:
        assert w == 2 and r == rank
        assert t == 11.0                      # the slowest rank's time
        assert n == 3000.0                    # whole-job trials
        assert win == 1 and abs(best - 0.6) < 1e-12 and c == [1.0] * 6   # every rank holds the winner


def test_single_rank_helpers_need_no_process_group():
    from powder6_b200.dist import best_over_ranks, max_over_ranks, sum_over_ranks
    assert max_over_ranks(3.5, 1) == 3.5 and sum_over_ranks(2.0, 1) == 2.0
    b, c, w = best_over_ranks(0.7, np.arange(3), 1)
    assert b == 0.7 and w == 0 and list(c) == [0, 1, 2]
