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


class FakeSession:
    """Stands in for WyckoffSession on the CPU: every chunk, replica i of
    assignment A reports best cc = base(rank, A) + a small generation term,
    so rank (A mod 2) holds the best structure of assignment A.  Coordinates
    encode (rank, A) so the test can see whose structure won."""

    def __init__(self, problem, n, rank):
        self.problem, self.num_particles, self.rank = problem, n, rank
        self.coords_per_particle = problem.max_sites * 3
        self.assign = np.zeros(n, dtype=np.uint32)
        self.g = 0
        self.launches = 0
        self.state = None

    def set_assign(self, a):
        self.assign = np.array(a, dtype=np.uint32)

    def set_ladders(self, *a):
        pass

    def set_schedule(self, *a):
        pass

    def set_quench(self, *a):
        pass

    def set_params(self, *a):
        pass

    def sync_state(self, pos, st):
        self.state = np.array(st)

    def run(self, g0, ng, swap, reeval):
        self.g = g0 + ng
        self.launches += 1

    def synchronize(self, timeout=60.0):
        pass

    def last_kernel_ms(self):
        return 1.0

    def launch_count(self):
        return self.launches

    def read_state(self):
        from powder6_b200.swarm_wyckoff import STATE_DTYPE
        n, cpp = self.num_particles, self.coords_per_particle
        st = np.zeros(n, dtype=STATE_DTYPE)
        A = self.assign.astype(np.int64)
        win = (A % 2) == self.rank
        st['best_fit'] = 0.0
        st['best_cc'] = np.where(win, 0.8, 0.5) + 1e-6 * self.g + 1e-9 * np.arange(n)
        st['best_pen'] = 0.0
        st['cc'] = st['best_cc']
        best = np.repeat((10.0 * self.rank + A + 0.5) / 100.0, cpp).astype(np.float32)
        return best.copy(), best, st


def _search_worker(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from powder6_b200.swarm_wyckoff import run_wyckoff_search
        from powder6_b200.workloads import wyckoff_problem
        alt = (('Pb', '4c'), ('S', '4c'), ('O', '8d'), ('O', '8d'))
        P = wyckoff_problem(seed=1, extra_assignments=[alt], contact_attempts=20)
        sess = FakeSession(P, 64, rank)
        stop_calls = []

        def should_stop():          # rank 1 asks to stop at its fourth check; both ranks must stop together
            stop_calls.append(1)
            return rank == 1 and len(stop_calls) >= 4
        res = run_wyckoff_search(P, 64, 100, restarts=1, seed=100 + rank, chunk=20, session=sess, world=world,
                                 do_quench=False, should_stop=should_stop)
        q.put((rank, {A: (round(b['cc'], 9), b['coords'][:3].tolist()) for A, b in res.bests.items()},
               res.best_assignment, sess.launches))
    finally:
        dist.destroy_process_group()


def test_sharded_search_every_rank_ends_with_the_global_winners():
    world = 2
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_search_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, b0, w0, l0), (_, b1, w1, l1) = out
    assert b0 == b1 and w0 == w1                  # the same per-assignment winners on both ranks
    # assignment 0's best came from rank 0, assignment 1's from rank 1 (coordinates encode the rank)
    assert b0[0][1][0] == pytest.approx(0.005) and b0[1][1][0] == pytest.approx(0.115)
    # the stop asked by rank 1 after three chunks reached both ranks before their fourth launch
    assert l0 == l1 == 3
