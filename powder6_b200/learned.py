"""Learned-proposal Wyckoff search.

The plain search (js/swarm_wyckoff.js, swarm_reflection.wgsl:657-725) draws
one random move per replica per generation.  Here a small network -- three
layers, width 256, bf16 weights at inference -- is trained on the GPU by the
project's own kernels (``p6_mlp_*``) on the moves the plain search itself
made: the 64 features of each move (which site, where it was, where it went,
the step, the replica's state) and the fitness change the exact evaluation
gave it.  The learned search then draws K candidate moves per replica, lets
the network rank them by predicted gain, and evaluates the best one with the
exact structure-factor fitness, which alone decides the Metropolis
acceptance (``p6_wy_learned_step``).  With K = 1 and no network the same
loop is the plain search, which is also how the training records are
collected.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import _lib
from ._lib import check, ptr
from .swarm_wyckoff import (SW_DEFAULTS, WyckoffSession, build_ladders, initial_state, project_all, schedule)
from .workloads import WyckoffProblem, mulberry32, wyckoff_problem

N_FEATURES = 64


class ProposalNet:
    """p6_mlp: d_in -> width -> width -> d_out, ReLU."""

    def __init__(self, d_in: int = N_FEATURES, width: int = 256, d_out: int = 1, seed: int = 1, device: int = 0):
        self.lib = _lib.load()
        self.d_in, self.width, self.d_out = d_in, width, d_out
        h = C.c_void_p()
        check(self.lib.p6_mlp_create(d_in, width, d_out, seed, device, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, 'h', None):
            self.lib.p6_mlp_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        n = C.c_longlong()
        check(self.lib.p6_mlp_params(self.h, None, None, C.byref(n)))
        out = np.zeros(n.value, dtype=np.float32)
        check(self.lib.p6_mlp_params(self.h, ptr(out), None, None))
        return out

    def set_params(self, w: np.ndarray):
        w = np.ascontiguousarray(w, dtype=np.float32)
        check(self.lib.p6_mlp_params(self.h, None, ptr(w), None))

    def gradients(self, X, T, mask=None):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32).reshape(len(X), self.d_out)
        M = None if mask is None else np.ascontiguousarray(mask, dtype=np.float32).reshape(len(X), self.d_out)
        g = np.zeros(len(self.params()), dtype=np.float32)
        loss = C.c_float()
        check(self.lib.p6_mlp_gradients(self.h, ptr(X), ptr(T), None if M is None else ptr(M), len(X), ptr(g),
                                        C.byref(loss)))
        return g, loss.value

    def train(self, X, T, mask=None, epochs: int = 10, batch: int = 1024, lr: float = 1e-3, seed: int = 1):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32).reshape(len(X), self.d_out)
        M = None if mask is None else np.ascontiguousarray(mask, dtype=np.float32).reshape(len(X), self.d_out)
        losses = np.zeros(epochs, dtype=np.float32)
        check(self.lib.p6_mlp_train(self.h, ptr(X), ptr(T), None if M is None else ptr(M), len(X), int(epochs),
                                    int(batch), float(lr), int(seed), ptr(losses)))
        return losses

    def predict(self, X) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.zeros((len(X), self.d_out), dtype=np.float32)
        check(self.lib.p6_mlp_predict(self.h, ptr(X), len(X), ptr(Y)))
        return Y


def learned_step(sess: WyckoffSession, net: Optional[ProposalNet], K: int, gen: int, reeval: bool,
                 records: bool = False, swap_every: int = int(SW_DEFAULTS['swapEvery'])):
    """One generation through p6_wy_learned_step; with ``records`` returns
    (features, gains, accepted, predicted) of the evaluated proposals."""
    n = sess.num_particles
    if records:
        X = np.zeros((n, N_FEATURES), dtype=np.float32)
        g = np.zeros(n, dtype=np.float32)
        a = np.zeros(n, dtype=np.float32)
        sc = np.zeros(n, dtype=np.float32)
        check(sess.lib.p6_wy_learned_step(sess.h, None if net is None else net.h, int(K), int(gen), int(swap_every),
                                          1 if reeval else 0, ptr(X), ptr(g), ptr(a), ptr(sc)))
        return X, g, a, sc
    check(sess.lib.p6_wy_learned_step(sess.h, None if net is None else net.h, int(K), int(gen), int(swap_every),
                                      1 if reeval else 0, None, None, None, None))
    return None


def learned_problem(seed: int = 1, dmin: float = 1.5) -> WyckoffProblem:
    """P2_1/c, a = 10.2, b = 12.1, c = 15.3 A, beta = 100 deg; 17 non-H atoms
    of C10N6S on general positions (4e), 68 atoms per cell; d_min 1.5 A.
    The atoms are independent sites (no rigid fragment or torsions: the
    reference describes molecules by distance rules on general positions)."""
    cell = {'a': 10.2, 'b': 12.1, 'c': 15.3, 'alpha': 90.0, 'beta': 100.0, 'gamma': 90.0}
    sites = [('C', '4e')] * 10 + [('N', '4e')] * 6 + [('S', '4e')]
    return wyckoff_problem(seed=seed, group_number=14, cell=cell, composition=(('C', 40), ('N', 24), ('S', 4)),
                           sites=tuple(sites), dmin=dmin, true_min_contact=1.1, contact_attempts=200)


def start(sess: WyckoffSession, problem: WyckoffProblem, generations: int, seed: int,
          settings: Optional[dict] = None):
    """Ladders, schedule and a seeded random start for a learned or plain run."""
    d = dict(SW_DEFAULTS)
    d.update(settings or {})
    n = sess.num_particles
    assign = np.zeros(n, dtype=np.uint32)
    sess.set_assign(assign)
    ladders, temps = build_ladders(assign, int(d['rungs']), d['tempCold'], d['tempHot'])
    sess.set_ladders(ladders, int(d['rungs']))
    groups, pen = schedule(generations, problem.refl.n_groups, d)
    sess.set_schedule(groups, pen)
    rnd = mulberry32(seed)
    pos = project_all(problem, np.array([rnd() for _ in range(n * sess.coords_per_particle)], dtype=np.float32),
                      assign)
    sess.sync_state(pos, initial_state(n, temps, rnd, d))
    return groups, pen


def collect_records(sess: WyckoffSession, problem: WyckoffProblem, generations: int, seed: int,
                    every: int = 1):
    """Plain search (K = 1, no network) with the records of every ``every``-th
    generation: the training data."""
    groups, _ = start(sess, problem, generations, seed)
    Xs, gs, acc = [], [], []
    for g in range(generations):
        reeval = g == 0 or groups[g] != groups[g - 1]
        if g % every == 0:
            X, gain, a, _ = learned_step(sess, None, 1, g, reeval, records=True)
            ok = np.isfinite(gain)
            Xs.append(X[ok]); gs.append(gain[ok]); acc.append(a[ok])
        else:
            learned_step(sess, None, 1, g, reeval)
    return np.concatenate(Xs), np.concatenate(gs), np.concatenate(acc)


def gain_targets(gains: np.ndarray):
    """Fitness changes scaled to unit spread and clipped at +/-5 (the network's target)."""
    s = float(np.std(gains)) or 1.0
    return np.clip(gains / s, -5.0, 5.0).astype(np.float32), s


@dataclass
class SearchTrace:
    seconds: List[float] = field(default_factory=list)
    best_cc: List[float] = field(default_factory=list)
    generations: int = 0
    time_to_target: Optional[float] = None
    device_ms: float = 0.0


def run(sess: WyckoffSession, problem: WyckoffProblem, generations: int, seed: int, net: Optional[ProposalNet] = None,
        K: int = 8, check_every: int = 50, target_cc: Optional[float] = None) -> SearchTrace:
    """A search of ``generations`` generations, learned (net, K) or plain
    (net None, K 1), timing the best cc every ``check_every`` generations."""
    groups, _ = start(sess, problem, generations, seed)
    tr = SearchTrace()
    sess.synchronize(60)
    t0 = time.perf_counter()
    check(sess.lib.p6_wy_time_mark(sess.h, 0))
    k = K if net is not None else 1
    for g in range(generations):
        reeval = g == 0 or groups[g] != groups[g - 1]
        learned_step(sess, net, k, g, reeval)
        if (g + 1) % check_every == 0 or g + 1 == generations:
            _, _, st = sess.read_state()
            ok = st['best_fit'] > -1e29
            b = float(np.max(st['best_cc'][ok])) if np.any(ok) else float('nan')
            tr.seconds.append(time.perf_counter() - t0)
            tr.best_cc.append(b)
            if target_cc is not None and tr.time_to_target is None and b >= target_cc:
                tr.time_to_target = tr.seconds[-1]
    check(sess.lib.p6_wy_time_mark(sess.h, 1))
    sess.synchronize(600)
    tr.device_ms = sess.last_kernel_ms()
    tr.generations = generations
    return tr
