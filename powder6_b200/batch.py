"""Many independent Wyckoff searches in one persistent launch (p6_wy_batch_*).

The reference runs one search per worker (js/wyckoff_worker.js, one
``runWyckoffSearch`` each).  Here each search keeps its own session --
tables, replica state, ladders, schedule -- and ``WyckoffBatch`` runs all
their ladders in one launch of persistent CTAs that take (search, ladder)
items from a list, captured in a CUDA graph.  ``autotune`` picks the launch
shape (persistent CTAs per SM, item order) by timing a short probe of the
actual batch; ``run_batched`` sets the searches up, tunes, runs and reads
the per-search results.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check
from .swarm_wyckoff import WyckoffSession, build_ladders, initial_state, project_all, schedule, SW_DEFAULTS
from .workloads import BatchItem, mulberry32


class WyckoffBatch:
    def __init__(self, sessions: Sequence[WyckoffSession]):
        self.lib = _lib.load()
        self.sessions = list(sessions)
        arr = (C.c_void_p * len(self.sessions))(*[s.h.value for s in self.sessions])
        self._arr = arr
        h = C.c_void_p()
        check(self.lib.p6_wy_batch_create(arr, len(self.sessions), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, 'h', None):
            self.lib.p6_wy_batch_destroy(self.h)
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

    def set_launch(self, ctas_per_sm: int = 0, order: int = 0):
        check(self.lib.p6_wy_batch_set_launch(self.h, int(ctas_per_sm), int(order)))

    def query(self) -> dict:
        m, sm, it, ln = C.c_int(), C.c_int(), C.c_int(), C.c_longlong()
        check(self.lib.p6_wy_batch_query(self.h, C.byref(m), C.byref(sm), C.byref(it), C.byref(ln)))
        return {'max_ctas_per_sm': m.value, 'smem_bytes': sm.value, 'items': it.value, 'launches': ln.value}

    def run(self, gen0: Sequence[int], n_gen: Sequence[int], swap_every: int, reeval_first: bool = True,
            use_graph: bool = True):
        g0 = np.ascontiguousarray(gen0, dtype=np.int32)
        ng = np.ascontiguousarray(n_gen, dtype=np.int32)
        self._keep = (g0, ng)
        check(self.lib.p6_wy_batch_run(self.h, g0.ctypes.data, ng.ctypes.data, int(swap_every),
                                       1 if reeval_first else 0, 1 if use_graph else 0))

    def synchronize(self, timeout: float = 600.0):
        check(self.lib.p6_wy_batch_synchronize(self.h, float(timeout)))

    def last_ms(self) -> float:
        v = C.c_float()
        check(self.lib.p6_wy_batch_last_ms(self.h, C.byref(v)))
        return v.value


@dataclass
class BatchSetup:
    sessions: List[WyckoffSession]
    starts: List[tuple]          # (positions, state) per search
    generations: List[int]


def setup_searches(items: Sequence[BatchItem], generations: int = 2000, seed: int = 1,
                   settings: Optional[dict] = None) -> BatchSetup:
    """One session per search: one assignment, ladders of 8, the resolution and
    penalty ramps over ``generations``, seeded random starts (not yet uploaded)."""
    d = dict(SW_DEFAULTS)
    d.update(settings or {})
    sessions, starts, gens = [], [], []
    for k, it in enumerate(items):
        P = it.problem
        s = WyckoffSession(P, it.replicas, run_key=seed * 1000 + k, cos_mode=0, settings=settings,
                               incremental=0)
        n = s.num_particles
        assign = np.zeros(n, dtype=np.uint32)
        s.set_assign(assign)
        ladders, temps = build_ladders(assign, int(d['rungs']), d['tempCold'], d['tempHot'])
        s.set_ladders(ladders, int(d['rungs']))
        g, pen = schedule(generations, P.refl.n_groups, d)
        s.set_schedule(g, pen)
        rnd = mulberry32(seed * 7919 + k)
        pos = project_all(P, np.array([rnd() for _ in range(n * s.coords_per_particle)], dtype=np.float32), assign)
        st = initial_state(n, temps, rnd, d)
        sessions.append(s)
        starts.append((pos, st))
        gens.append(generations)
    return BatchSetup(sessions, starts, gens)


def reset(setup: BatchSetup):
    for s, (pos, st) in zip(setup.sessions, setup.starts):
        s.sync_state(pos, st)


def autotune(batch: WyckoffBatch, setup: BatchSetup, probe: int = 40) -> dict:
    """Times every launch shape (persistent CTAs per SM x item order) on the
    first ``probe`` generations of the batch and keeps the fastest."""
    q = batch.query()
    trials = []
    n = len(setup.sessions)
    for per_sm in range(1, q['max_ctas_per_sm'] + 1):
        for order in (0, 1):
            reset(setup)
            batch.set_launch(per_sm, order)
            batch.run([0] * n, [min(probe, g) for g in setup.generations], int(SW_DEFAULTS['swapEvery']), True,
                      use_graph=False)
            batch.synchronize()
            trials.append((batch.last_ms(), per_sm, order))
    best = min(trials)
    batch.set_launch(best[1], best[2])
    return {'ctas_per_sm': best[1], 'order': best[2], 'probe_ms': best[0],
            'trials': [{'ms': t, 'ctas_per_sm': p, 'order': o} for t, p, o in trials]}


def read_results(setup: BatchSetup) -> List[dict]:
    out = []
    for s in setup.sessions:
        _, best, st = s.read_state()
        ok = st['best_fit'] > -1e29
        i = int(np.argmax(np.where(ok, st['best_cc'], -np.inf))) if np.any(ok) else 0
        out.append({'best_cc': float(st['best_cc'][i]) if np.any(ok) else float('nan'),
                    'accepted': int(st['accepted'].sum()),
                    'coords': best[i * s.coords_per_particle:(i + 1) * s.coords_per_particle].copy()})
    return out


def run_batched(items: Sequence[BatchItem], generations: int = 2000, seed: int = 1, tune: bool = True,
                use_graph: bool = True, settings: Optional[dict] = None) -> dict:
    """Set up, tune, run all searches to ``generations`` in one launch; returns
    the per-search results, the device time, the tuning record and the trials."""
    setup = setup_searches(items, generations, seed, settings)
    try:
        with WyckoffBatch(setup.sessions) as b:
            tuning = autotune(b, setup) if tune else None
            reset(setup)
            n = len(setup.sessions)
            b.run([0] * n, setup.generations, int(SW_DEFAULTS['swapEvery']), True, use_graph=use_graph)
            b.synchronize()
            ms = b.last_ms()
            info = b.query()
        results = read_results(setup)
        trials = int(sum(s.num_particles * g for s, g in zip(setup.sessions, setup.generations)))
        return {'results': results, 'ms': ms, 'tuning': tuning, 'trials': trials, 'query': info}
    finally:
        for s in setup.sessions:
            s.close()
