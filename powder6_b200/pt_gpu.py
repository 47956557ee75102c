"""Parallel-tempering backend on the B200, mirroring RVPTGPU (js/pt_gpu.js).

``compile(ctx)``, ``create(ctx)`` and ``run(ctx)`` keep the reference's call
surface (js/pt_gpu.js:20-227, 371-406, 409-423):

* ``compile`` builds the plan -- the reflections of the phase over the cell
  envelope (the upper bounds of the refined cell), the coset representatives,
  the atoms and the observed pattern;
* ``create`` returns an object with ``plan``, ``close()``, ``initial(vectors)``,
  ``costs(vectors)`` and ``batch(count, bootstrap)`` (the state in the
  reference layout, chains x (3 nv + 12) floats);
* ``run`` validates two probes against ``ctx.cost`` (relative error 1e-3, a
  disagreement raises with "disagrees" in the message, as js/pt_gpu.js:413-415),
  runs ``ctx.setup.sweeps`` sweeps in batches of ceil(8 / nv), re-scores every
  new per-chain best with ``ctx.cost`` and returns ``{x, stopped, pt}``.

Any failure raises; the caller falls back to its CPU tempering, as
RVCore.refineAsync does (js/rietveld_core.js:2450-2467).

``ctx`` is a ``PTContext``: the problem (``PTProblem``), the start ``x``, the
per-parameter bounds ``info``, ``setup`` {sweeps, chains, maxTemp, seed,
initialCost, scales}, and the callables ``cost``, ``feasible``, ``should_stop``,
``on_iter``.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import P6PtProblem, check
from .reflections import generate_reflections
from .symmetry import cosets, space_group

# Full parameter vector layout shared with the kernel.
FULL_NAMES = ['scale', 'a', 'b', 'c', 'alpha', 'beta', 'gamma', 'U', 'V', 'W', 'X', 'Y', 'zero', 'Biso']
PROFILE_WINDOW_MAX_DEG = 10.0


@dataclass
class PTProblem:
    group_number: int
    system: str
    atoms: List[dict]                 # {element, pos (3), mult, occ, a (5), b (5), c}
    tth: np.ndarray
    y: np.ndarray
    w: np.ndarray
    lambda1: float
    lambda2: float
    ratio: float
    pol_k: float
    min_fwhm: float
    n_bkg: int
    values: np.ndarray                # full parameter vector
    refined: List[str]                # names of the refined parameters
    lo: np.ndarray
    hi: np.ndarray
    # March-Dollase preferred orientation (js/rietveld_core.js:824-853): the
    # reciprocal-lattice direction, or None (off).  Its parameter 'po' (r) is
    # the entry of the full vector after the background.
    po_dir: Optional[Sequence[float]] = None
    # SL/HL axial-divergence asymmetry of the TCH profile (js/profile.js:608-617):
    # when True, 'SL' and 'HL' are the full-vector entries after the background
    # (and after 'po').
    asym: bool = False
    # Phase method (js/rietveld_core.js:110, js/pt_gpu.js:259-297): 'rietveld'
    # takes the heights from the structure; 'lebail' and 'wppf' leave every
    # reflection's height free and non-negative, solved per evaluation by NNLS
    # against the observed pattern minus the background (atoms unused; at most
    # 64 reflections in the envelope).
    method: str = 'rietveld'
    # Sample displacement and transparency (js/pt_gpu.js:169-171, :355): when
    # True, 'disp' and 'transp' are the full-vector entries after SL, HL (or
    # after 'po', or after the background).
    shift: bool = False

    @property
    def method_code(self) -> int:
        if self.method == 'rietveld':
            return 0
        if self.method in ('lebail', 'wppf'):
            return 1
        raise ValueError(f"method must be 'rietveld', 'lebail' or 'wppf', not {self.method!r}")

    @property
    def index(self) -> np.ndarray:
        return np.array([self.full_index(n) for n in self.refined], dtype=np.int32)

    def full_index(self, name: str) -> int:
        if name.startswith('bkg'):
            return len(FULL_NAMES) + int(name[3:])
        if name == 'po':
            if self.po_dir is None:
                raise KeyError('po: the problem has no preferred-orientation direction')
            return len(FULL_NAMES) + self.n_bkg
        if name in ('SL', 'HL'):
            if not self.asym:
                raise KeyError(f'{name}: the problem has no asymmetry')
            return len(FULL_NAMES) + self.n_bkg + (1 if self.po_dir is not None else 0) + (name == 'HL')
        if name in ('disp', 'transp'):
            if not self.shift:
                raise KeyError(f'{name}: the problem has no sample shift')
            return (len(FULL_NAMES) + self.n_bkg + (1 if self.po_dir is not None else 0) + (2 if self.asym else 0) +
                    (name == 'transp'))
        return FULL_NAMES.index(name)

    def apply(self, x: Sequence[float]) -> np.ndarray:
        v = self.values.astype(np.float64).copy()
        for j, i in enumerate(self.index):
            v[i] = x[j]
        if self.system == 'cubic':
            v[2] = v[3] = v[1]
        return v


@dataclass
class PTContext:
    problem: PTProblem
    x: np.ndarray
    setup: dict
    cost: Optional[Callable[[np.ndarray], float]] = None
    feasible: Optional[Callable[[np.ndarray], bool]] = None
    should_stop: Optional[Callable[[], bool]] = None
    on_iter: Optional[Callable[[dict], None]] = None
    max_iter: int = 0


def reflection_dmin(problem: PTProblem) -> float:
    """reflectionDmin with the envelope of the zero-point range (js/rietveld_core.js:238-245)."""
    lam = problem.lambda1
    if problem.ratio > 1e-6 and problem.lambda2 > 0:
        lam = min(lam, problem.lambda2)
    def magnitude(name):
        v = abs(problem.values[problem.full_index(name)])
        if name in problem.refined:
            j = problem.refined.index(name)
            v = max(abs(problem.lo[j]), abs(problem.hi[j]))
        return v
    margin = PROFILE_WINDOW_MAX_DEG + magnitude('zero')
    if problem.shift:
        margin += (magnitude('disp') * 0.001 + magnitude('transp')) * 180.0 / math.pi
    upper = min(179.999999, float(problem.tth[-1]) + margin + .001)
    return lam / (2 * math.sin(math.radians(upper) / 2))


@dataclass
class Plan:
    hkl: np.ndarray
    mult: np.ndarray
    rep_rot: np.ndarray
    rep_trans: np.ndarray
    dmin: float
    nv: int
    chains: int
    stride: int
    point_count: int
    reflection_count: int
    eq_start: Optional[np.ndarray] = None   # March-Dollase: equivalents of each reflection
    eq_hkl: Optional[np.ndarray] = None


def compile(ctx: PTContext) -> Plan:
    """The packed plan (js/pt_gpu.js:20-227): envelope reflections, cosets."""
    P = ctx.problem
    g = space_group(P.group_number)
    dmin = reflection_dmin(P)
    v = P.values.copy()
    # envelope: the largest cell the bounds allow (monotone for the orthogonal and cubic metrics)
    for name in ('a', 'b', 'c'):
        if name in P.refined:
            v[P.full_index(name)] = P.hi[P.refined.index(name)]
    if P.system == 'cubic':
        v[2] = v[3] = v[1]
    cell = {'a': v[1], 'b': v[2], 'c': v[3], 'alpha': v[4], 'beta': v[5], 'gamma': v[6]}
    refl = generate_reflections(cell, g.ops, dmin, with_eq=P.po_dir is not None)
    if not refl:
        raise RuntimeError('No reflections for the PT backend.')
    reps, _nc = cosets(g.ops)
    hkl = np.array([[r.h, r.k, r.l] for r in refl], dtype=np.int32)
    mult = np.array([r.m for r in refl], dtype=np.int32)
    rep_rot = np.array([o.r for o in reps], dtype=np.int32)
    rep_trans = np.array([o.t_frac for o in reps], dtype=np.float64)
    nv = len(P.refined)
    eq_start = eq_hkl = None
    if P.po_dir is not None:
        counts = np.array([len(r.eq) for r in refl], dtype=np.int32)
        eq_start = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
        eq_hkl = np.concatenate([np.asarray(r.eq, dtype=np.int32).reshape(-1, 3) for r in refl]).astype(np.int32)
    return Plan(hkl, mult, rep_rot, rep_trans, dmin, nv, int(ctx.setup['chains']), 3 * nv + 12, len(P.tth), len(refl),
                eq_start, eq_hkl)


class PTSession:
    """create(ctx) (js/pt_gpu.js:371-406): device state of one PT run."""

    def __init__(self, ctx: PTContext, device: int = 0, plan: Optional[Plan] = None):
        self.lib = _lib.load()
        self.ctx = ctx
        self.plan = plan or compile(ctx)
        P = ctx.problem
        self._keep = []

        def a(x, dt):
            x = np.ascontiguousarray(x, dtype=dt)
            self._keep.append(x)
            return x.ctypes.data

        n_reps = len(self.plan.rep_rot)
        pr = P6PtProblem()
        pr.n_refl = self.plan.reflection_count
        pr.hkl = a(self.plan.hkl, np.int32)
        pr.mult = a(self.plan.mult, np.int32)
        pr.n_reps = n_reps
        pr.rep_rot = a(self.plan.rep_rot, np.int32)
        pr.rep_trans = a(self.plan.rep_trans, np.float64)
        pr.n_atoms = len(P.atoms)
        pr.atom_pos = a([at['pos'] for at in P.atoms], np.float64)
        pr.atom_wmult = a([at['mult'] / n_reps for at in P.atoms], np.float64)
        pr.atom_occ = a([at.get('occ', 1.0) for at in P.atoms], np.float64)
        pr.ff_a = a([at['a'] for at in P.atoms], np.float64)
        pr.ff_b = a([at['b'] for at in P.atoms], np.float64)
        pr.ff_c = a([at['c'] for at in P.atoms], np.float64)
        pr.n_points = len(P.tth)
        pr.tth = a(P.tth, np.float64)
        pr.y = a(P.y, np.float64)
        pr.w = a(P.w, np.float64)
        pr.lambda1, pr.lambda2, pr.ratio, pr.pol_k = P.lambda1, P.lambda2, P.ratio, P.pol_k
        pr.min_fwhm = P.min_fwhm
        pr.dmin = self.plan.dmin
        pr.n_bkg = P.n_bkg
        pr.n_full = len(P.values)
        pr.full_values = a(P.values, np.float64)
        pr.nv = self.plan.nv
        pr.index = a(P.index, np.int32)
        pr.lo = a(P.lo, np.float64)
        pr.hi = a(P.hi, np.float64)
        pr.scales = a(ctx.setup['scales'], np.float64)
        pr.cubic = 1 if P.system == 'cubic' else 0
        pr.chains = self.plan.chains
        pr.max_temp = float(ctx.setup['maxTemp'])
        pr.seed = int(ctx.setup['seed']) & 0xFFFFFFFF
        if P.po_dir is not None:
            pr.has_po = 1
            pr.eq_start = a(self.plan.eq_start, np.int32)
            pr.eq_hkl = a(self.plan.eq_hkl, np.int32)
            for i in range(3):
                pr.po_dir[i] = float(P.po_dir[i])
        pr.has_asym = 1 if P.asym else 0
        pr.method = P.method_code
        pr.has_shift = 1 if P.shift else 0
        h = C.c_void_p()
        check(self.lib.p6_pt_create(C.byref(pr), int(device), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, 'h', None):
            self.lib.p6_pt_destroy(self.h)
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

    def costs(self, vectors: Sequence[Sequence[float]], with_pattern: bool = False):
        v = np.ascontiguousarray(np.asarray(vectors, dtype=np.float64).reshape(-1, self.plan.nv))
        out = np.zeros(len(v), dtype=np.float64)
        y = np.zeros((len(v), self.plan.point_count), dtype=np.float32) if with_pattern else None
        check(self.lib.p6_pt_costs(self.h, v.ctypes.data, len(v), out.ctypes.data,
                                   None if y is None else y.ctypes.data))
        return (out, y) if with_pattern else out

    def costs_static(self, vectors: Sequence[Sequence[float]], with_pattern: bool = False):
        """costs() through p6_pt_costs_static: no device allocation, at most
        P6_PT_STATIC_SCRATCH_BYTES (4 MiB) of vectors, costs and patterns per call."""
        v = np.ascontiguousarray(np.asarray(vectors, dtype=np.float64).reshape(-1, self.plan.nv))
        out = np.zeros(len(v), dtype=np.float64)
        y = np.zeros((len(v), self.plan.point_count), dtype=np.float32) if with_pattern else None
        check(self.lib.p6_pt_costs_static(self.h, v.ctypes.data, len(v), out.ctypes.data,
                                          None if y is None else y.ctypes.data))
        return (out, y) if with_pattern else out

    def vector_capacity(self) -> int:
        """Vectors the allocating scratch of costs() holds (0 until costs() first runs)."""
        n = C.c_int(0)
        check(self.lib.p6_pt_vector_capacity(self.h, C.byref(n)))
        return int(n.value)

    def initial(self, vectors: Sequence[Sequence[float]]):
        v = np.ascontiguousarray(np.asarray(vectors, dtype=np.float64).reshape(-1, self.plan.nv))
        check(self.lib.p6_pt_initial(self.h, v.ctypes.data, len(v)))

    def batch(self, count: int, bootstrap: bool = False) -> np.ndarray:
        check(self.lib.p6_pt_batch(self.h, int(count), 1 if bootstrap else 0))
        return self.state()

    def launch(self, count: int, bootstrap: bool = False):
        check(self.lib.p6_pt_batch(self.h, int(count), 1 if bootstrap else 0))

    def state(self) -> np.ndarray:
        st = np.zeros(self.plan.chains * self.plan.stride, dtype=np.float32)
        check(self.lib.p6_pt_read_state(self.h, st.ctypes.data, None, None, None, None))
        return st

    def exact_state(self):
        c, nv = self.plan.chains, self.plan.nv
        x = np.zeros((c, nv))
        best = np.zeros((c, nv))
        costs = np.zeros((c, 2))
        counters = np.zeros((c, 4))
        check(self.lib.p6_pt_read_state(self.h, None, x.ctypes.data, best.ctypes.data, costs.ctypes.data,
                                        counters.ctypes.data))
        return x, best, costs, counters

    def set_trace(self, on: bool):
        check(self.lib.p6_pt_set_trace(self.h, 1 if on else 0))

    def read_trace(self):
        """Per chain, the last sweep's exchange {tried, swapped, la, log u} and
        moves (nv x {j, proposed x_j, log u, cost before, cost, accepted})."""
        c, nv = self.plan.chains, self.plan.nv
        out = np.zeros(c * (4 + 6 * nv), dtype=np.float64)
        check(self.lib.p6_pt_read_trace(self.h, out.ctypes.data))
        out = out.reshape(c, 4 + 6 * nv)
        return out[:, :4], out[:, 4:].reshape(c, nv, 6)

    def synchronize(self, timeout: float = 60.0):
        check(self.lib.p6_pt_synchronize(self.h, float(timeout)))

    # --- least-squares finish (FP64 on the device)
    def model_costs(self, vectors) -> np.ndarray:
        """chi^2 of each refined vector with the FP64 model (one launch)."""
        v = np.ascontiguousarray(np.asarray(vectors, dtype=np.float64).reshape(-1, self.plan.nv))
        out = np.zeros(len(v))
        check(self.lib.p6_pt_model_costs(self.h, v.ctypes.data, len(v), out.ctypes.data))
        return out

    def model_cost(self, x) -> float:
        return float(self.model_costs([x])[0])

    def normal(self, x):
        """(A = J'WJ, g = J'W r, f = chi^2) at x, FP64 on the device."""
        nv = self.plan.nv
        x = np.ascontiguousarray(x, dtype=np.float64)
        A = np.zeros((nv, nv))
        g = np.zeros(nv)
        f = C.c_double()
        check(self.lib.p6_pt_normal(self.h, x.ctypes.data, A.ctypes.data, g.ctypes.data, C.byref(f)))
        return A, g, f.value

    def linear_start(self, x):
        x = np.ascontiguousarray(np.array(x, dtype=np.float64))
        f = C.c_double()
        check(self.lib.p6_pt_linear_start(self.h, x.ctypes.data, C.byref(f)))
        return x, f.value

    def lm(self, x, max_iter: int = 20, tol: float = 1e-5):
        x = np.ascontiguousarray(np.array(x, dtype=np.float64))
        out = np.zeros(4)
        check(self.lib.p6_pt_lm(self.h, x.ctypes.data, int(max_iter), float(tol), out.ctypes.data))
        return x, {'chi2': out[0], 'iterations': int(out[1]), 'accepted': int(out[2]), 'code': int(out[3])}

    def last_batch_ms(self) -> float:
        v = C.c_float()
        check(self.lib.p6_pt_last_batch_ms(self.h, C.byref(v)))
        return v.value

    def launch_count(self) -> int:
        v = C.c_longlong()
        check(self.lib.p6_pt_launch_count(self.h, C.byref(v)))
        return v.value

    @property
    def split(self) -> int:
        """CTAs per chain in the sweeps (2: a two-CTA cluster per chain)."""
        v = C.c_int()
        check(self.lib.p6_pt_get_split(self.h, C.byref(v)))
        return v.value

    @split.setter
    def split(self, ctas_per_chain: int):
        check(self.lib.p6_pt_set_split(self.h, int(ctas_per_chain)))


def create(ctx: PTContext, device: int = 0) -> PTSession:
    return PTSession(ctx, device)


def _reflected(value, lo, hi):
    if math.isfinite(lo) and math.isfinite(hi):
        span = hi - lo
        if span <= 0:
            return lo
        folded = ((value - lo) % (2 * span) + 2 * span) % (2 * span)
        return lo + (folded if folded <= span else 2 * span - folded)
    return 2 * lo - value if value < lo else (2 * hi - value if value > hi else value)


def run(ctx: PTContext, device: int = 0, session: Optional[PTSession] = None) -> dict:
    """RVPTGPU.run (js/pt_gpu.js:409-423).

    ``ctx.cost`` re-scores the probes and each new per-chain best, as the
    reference does with its CPU model; when it is None, the session's FP64
    device model does both, with all the new bests of a batch in one launch.
    ``session`` reuses an open session (it is left open)."""
    P = ctx.problem
    gpu = session or create(ctx, device)
    try:
        x0 = np.asarray(ctx.x, dtype=np.float64)
        scales = np.asarray(ctx.setup['scales'], dtype=np.float64)
        probes = [x0, np.array([_reflected(v + s * 0.25, lo, hi) for v, s, lo, hi in zip(x0, scales, P.lo, P.hi)])]
        chains = int(ctx.setup['chains'])
        gc = gpu.costs([probes[c % 2] for c in range(chains)])
        ref = [ctx.cost(probes[0]), ctx.cost(probes[1])] if ctx.cost else list(gpu.model_costs(probes))
        validation = 0.0
        for c in range(chains):
            cpu = ref[c % 2]
            if not math.isfinite(cpu):
                continue
            err = abs(gc[c] - cpu) / max(1.0, cpu)
            validation = max(validation, err)
            if not math.isfinite(gc[c]) or err > 1e-3:
                raise RuntimeError(f'B200 PT cost disagrees with the double-precision model (relative error {err:.3g}).')
        gpu.initial([x0])
        gpu.batch(1, True)
        best = x0.copy()
        best_cost = float(ctx.setup.get('initialCost', ref[0]))
        seen = set()
        sweeps = int(ctx.setup['sweeps'])
        count = max(1, math.ceil(8 / len(x0)))
        completed = 0
        stopped = False
        while completed < sweeps:
            if ctx.should_stop and ctx.should_stop():
                stopped = True
                break
            n = min(count, sweeps - completed)
            gpu.launch(n)
            completed += n
            _, bests, costs, _ = gpu.exact_state()
            fresh = []
            for c in range(chains):
                cand = bests[c]
                key = cand.tobytes()
                if key in seen:
                    continue
                seen.add(key)
                if not all(lo <= v <= hi for v, lo, hi in zip(cand, P.lo, P.hi)):
                    continue
                if ctx.feasible and not ctx.feasible(cand):
                    continue
                fresh.append(cand)
            if fresh:
                values = [ctx.cost(c) for c in fresh] if ctx.cost else gpu.model_costs(fresh)
                for cand, value in zip(fresh, values):
                    if value < best_cost:
                        best, best_cost = cand.copy(), float(value)
            if ctx.on_iter:
                ctx.on_iter({'it': completed, 'chi2': best_cost, 'maxIter': ctx.max_iter, 'stage': 'pt',
                             'backend': 'cuda'})
        _, _, _, counters = gpu.exact_state()
        stats = {'accepted': float(counters[:, 0].sum()), 'proposals': float(counters[:, 1].sum()),
                 'swaps': float(counters[:, 2].sum()), 'swapAttempts': float(counters[:, 3].sum())}
        pt = {'backend': 'cuda', 'chains': chains, 'sweeps': completed, 'requestedSweeps': sweeps,
              'maxTemp': ctx.setup['maxTemp'], 'seed': ctx.setup['seed'],
              'initialChi2': ctx.setup.get('initialCost'), 'bestChi2': best_cost, 'validationError': validation}
        pt.update(stats)
        return {'x': best, 'stopped': stopped, 'pt': pt}
    finally:
        if session is None:
            gpu.close()


def rwp(problem: PTProblem, chi2: float) -> float:
    """Rwp = sqrt(chi^2 / sum w y^2) over the points with w > 0 (js/rietveld_core.js:1578-1608)."""
    m = problem.w > 0
    return float(np.sqrt(chi2 / np.sum(problem.w[m] * problem.y[m] ** 2)))


def refine(ctx: PTContext, device: int = 0, max_iter: int = 20, tol: float = 1e-5,
           target_chi2: Optional[float] = None, finish: bool = True) -> dict:
    """refine() with algorithm 'pt' (js/rietveld_core.js:2242-2300) on the device:
    one Gauss-Newton step on the scale and background, tempering from there
    (``run``), the tempering's best kept if it is no worse than the start,
    then the least-squares finish.  Returns x, chi2, Rwp, the PT record, the
    LM record, the wall time at the end of each stage and, with
    ``target_chi2``, the wall time at which the best chi^2 so far first
    reached it (checked after the linear start, after every batch of sweeps
    and after the finish).  ``finish`` False stops after the tempering (the
    least-squares finish is skipped), so the tempering's own progress can be
    timed."""
    import time
    t0 = time.perf_counter()
    hit = {'t': None}

    def note(chi2):
        if target_chi2 is not None and hit['t'] is None and chi2 <= target_chi2:
            hit['t'] = time.perf_counter() - t0

    with PTSession(ctx, device) as gpu:
        x, f = gpu.linear_start(ctx.x)
        note(f)
        t_lin = time.perf_counter() - t0
        user_iter = ctx.on_iter

        def on_iter(p):
            note(p['chi2'])
            if user_iter:
                user_iter(p)
        setup = dict(ctx.setup)
        setup['initialCost'] = f
        sub = PTContext(ctx.problem, x, setup, cost=ctx.cost, feasible=ctx.feasible, should_stop=ctx.should_stop,
                        on_iter=on_iter, max_iter=ctx.max_iter)
        r = run(sub, device, session=gpu)
        t_pt = time.perf_counter() - t0
        if r['pt']['bestChi2'] <= f:
            x = r['x']
        if finish:
            xf, lm = gpu.lm(x, max_iter, tol)
            note(lm['chi2'])
        else:
            xf, lm = x, {'chi2': min(f, r['pt']['bestChi2']), 'skipped': True}
        t_lm = time.perf_counter() - t0
    return {'x': xf, 'chi2': lm['chi2'], 'rwp': rwp(ctx.problem, lm['chi2']), 'pt': r['pt'], 'lm': lm,
            'stopped': r['stopped'], 'seconds': {'linear': t_lin, 'pt': t_pt, 'lm': t_lm},
            'time_to_target': hit['t']}


# ---------------------------------------------------------------------------
# The NaCl parallel-tempering workload (seeded, synthetic).
# ---------------------------------------------------------------------------
FULLPROF_TO_GSAS_U = 1803.4     # 100^2 / (8 ln 2), Kaduk & Reid (2011)


def nacl_problem(seed: int = 1, tth0: float = 10.0, tth1: float = 120.0, step: float = 0.02,
                 peak_counts: float = 1e4, n_bkg: int = 6) -> PTProblem:
    """Fm-3m NaCl, a = 5.640 A, Na 4a, Cl 4b, Biso 1.0; Cu K-alpha-1/2 1.5406/1.5444,
    ratio 0.5; TCH U, V, W = 0.004, -0.002, 0.003 deg^2 and X (strain), Y (size)
    = 0.02, 0.01 deg in FullProf units, converted to the reference's GSAS units
    (GU = 1803.4 U; size -> X = 100 Y_FP; strain -> Y = 100 X_FP).  The observed
    pattern is left empty: ``synthesise`` fills it (Poisson counts, w = 1/max(1, y))."""
    from .workloads import load_form_factor_table
    ff = load_form_factor_table()
    n = int(round((tth1 - tth0) / step)) + 1
    tth = tth0 + step * np.arange(n, dtype=np.float64)
    atoms = []
    for el, pos in (('Na', (0.0, 0.0, 0.0)), ('Cl', (0.5, 0.5, 0.5))):
        e = ff[el]
        atoms.append({'element': el, 'pos': pos, 'mult': 4, 'occ': 1.0, 'a': e['a'], 'b': e['b'], 'c': e['c']})
    vals = np.zeros(len(FULL_NAMES) + n_bkg)
    vals[:len(FULL_NAMES)] = [1.0, 5.640, 5.640, 5.640, 90, 90, 90,
                              FULLPROF_TO_GSAS_U * 0.004, FULLPROF_TO_GSAS_U * -0.002, FULLPROF_TO_GSAS_U * 0.003,
                              100 * 0.01, 100 * 0.02, 0.0, 1.0]
    vals[len(FULL_NAMES):] = [300.0, -80.0, 40.0, -15.0, 8.0, -3.0][:n_bkg]
    refined = ['scale', 'a', 'Biso', 'U', 'V', 'W', 'zero']
    prob = PTProblem(225, 'cubic', atoms, tth, np.zeros(n), np.ones(n), 1.5406, 1.5444, 0.5, 1.0,
                     max(1e-4, 2 * step), n_bkg, vals, refined, np.zeros(7), np.zeros(7))
    prob.peak_counts = peak_counts
    prob.seed = seed
    return prob


def with_preferred_orientation(prob: PTProblem, direction: Sequence[float], r: float = 1.0, refine: bool = True,
                               lo: float = 0.5, hi: float = 2.0) -> PTProblem:
    """A copy of ``prob`` with March-Dollase preferred orientation along the
    reciprocal-lattice ``direction`` (js/rietveld_core.js:824-853): the March
    parameter r is appended to the full vector after the background and, with
    ``refine``, to the refined parameters with the bounds [lo, hi]."""
    import copy
    out = copy.copy(prob)
    out.po_dir = tuple(float(v) for v in direction)
    out.values = np.concatenate([np.asarray(prob.values, dtype=np.float64)[:len(FULL_NAMES) + prob.n_bkg], [r]])
    if refine:
        out.refined = list(prob.refined) + ['po']
        out.lo = np.concatenate([np.asarray(prob.lo, dtype=np.float64), [lo]])
        out.hi = np.concatenate([np.asarray(prob.hi, dtype=np.float64), [hi]])
    return out


def with_asymmetry(prob: PTProblem, SL: float = 0.0, HL: float = 0.0, refine: Sequence[str] = ('SL', 'HL'),
                   bounds: Optional[Dict[str, tuple]] = None) -> PTProblem:
    """A copy of ``prob`` with the SL/HL asymmetry (js/profile.js:608-617):
    SL and HL are appended to the full vector (after the background and any
    'po') and the names in ``refine`` to the refined parameters, with
    ``bounds`` (default SL [0, 0.05], HL [-0.05, 0.05])."""
    import copy
    b = {'SL': (0.0, 0.05), 'HL': (-0.05, 0.05)}
    b.update(bounds or {})
    out = copy.copy(prob)
    out.asym = True
    n0 = len(FULL_NAMES) + prob.n_bkg + (1 if prob.po_dir is not None else 0)
    out.values = np.concatenate([np.asarray(prob.values, dtype=np.float64)[:n0], [SL, HL]])
    out.refined = list(prob.refined) + list(refine)
    out.lo = np.concatenate([np.asarray(prob.lo, dtype=np.float64), [b[n][0] for n in refine]])
    out.hi = np.concatenate([np.asarray(prob.hi, dtype=np.float64), [b[n][1] for n in refine]])
    return out


def with_sample_shift(prob: PTProblem, disp: float = 0.0, transp: float = 0.0,
                      refine: Sequence[str] = ('disp', 'transp'), bounds: Optional[Dict[str, tuple]] = None) -> PTProblem:
    """A copy of ``prob`` with sample displacement and transparency
    (js/pt_gpu.js:169-171, :355): 'disp' and 'transp' appended to the full
    vector (after the background, 'po', SL and HL) and the names in
    ``refine`` to the refined parameters, with ``bounds`` (default disp
    [-100, 100], transp [-0.01, 0.01])."""
    import copy
    b = {'disp': (-100.0, 100.0), 'transp': (-0.01, 0.01)}
    b.update(bounds or {})
    out = copy.copy(prob)
    out.shift = True
    n0 = (len(FULL_NAMES) + prob.n_bkg + (1 if prob.po_dir is not None else 0) + (2 if prob.asym else 0))
    out.values = np.concatenate([np.asarray(prob.values, dtype=np.float64)[:n0], [disp, transp]])
    out.refined = list(prob.refined) + list(refine)
    out.lo = np.concatenate([np.asarray(prob.lo, dtype=np.float64), [b[n][0] for n in refine]])
    out.hi = np.concatenate([np.asarray(prob.hi, dtype=np.float64), [b[n][1] for n in refine]])
    return out


def set_bounds(prob: PTProblem, truth: np.ndarray):
    t = {n: truth[prob.full_index(n)] for n in prob.refined}
    lo = {'scale': 0.5 * t['scale'], 'a': 0.98 * t['a'], 'Biso': 0.0, 'U': 0.0, 'V': -20.0, 'W': 0.0, 'zero': -0.1}
    hi = {'scale': 1.5 * t['scale'], 'a': 1.02 * t['a'], 'Biso': 4.0, 'U': 40.0, 'V': 20.0, 'W': 30.0, 'zero': 0.1}
    prob.lo = np.array([lo[n] for n in prob.refined])
    prob.hi = np.array([hi[n] for n in prob.refined])


def synthesise(prob: PTProblem, pattern: Callable[[PTProblem, np.ndarray], np.ndarray], seed: int = 1):
    """Fill y, w with Poisson counts of the model at the true values, scaled so the
    strongest point is ~prob.peak_counts; returns the true refined vector."""
    rng = np.random.default_rng(seed)
    truth = prob.values.copy()
    bk = truth.copy()
    bk[0] = 0.0
    y_bkg = pattern(prob, bk)
    y1 = pattern(prob, truth)
    peak = float(np.max(y1 - y_bkg))
    truth[0] = (getattr(prob, 'peak_counts', 1e4) - float(np.max(y_bkg))) / max(peak, 1e-30)
    yc = pattern(prob, truth)
    y = rng.poisson(np.maximum(yc, 0)).astype(np.float64)
    prob.values = truth
    prob.y = y
    prob.w = 1.0 / np.maximum(1.0, y)
    set_bounds(prob, truth)
    return np.array([truth[prob.full_index(n)] for n in prob.refined])


def start_vectors(prob: PTProblem, truth_x: np.ndarray, n: int, seed: int = 1) -> List[np.ndarray]:
    """Uniform +/-5 % starts around the truth (the zero point, true value 0, by +/-0.01 deg)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        x = truth_x.copy()
        for j, name in enumerate(prob.refined):
            x[j] = truth_x[j] + (rng.uniform(-0.01, 0.01) if name == 'zero' else truth_x[j] * rng.uniform(-0.05, 0.05))
            x[j] = min(max(x[j], prob.lo[j]), prob.hi[j])
        out.append(x)
    return out


STEP_CAP = {'scale': None, 'a': 'cell', 'Biso': 2.0, 'U': 'profile', 'V': 'profile', 'W': 'profile', 'zero': 0.1,
            'po': 0.25, 'SL': 0.01, 'HL': 0.01, 'disp': 2.0, 'transp': 0.01}


def natural_scales(prob: PTProblem, x: np.ndarray) -> np.ndarray:
    """The 'natural' step of preparePT (0.15 stepCap, js/rietveld_core.js:2158-2164 and
    :511-524); with the curvature term the caller's J'WJ diagonal may shrink it."""
    out = np.zeros(len(x))
    for j, name in enumerate(prob.refined):
        cap = STEP_CAP.get(name)
        if cap == 'cell':
            cap = 0.02 * abs(x[j]) + 1e-6
        elif cap == 'profile':
            cap = 0.5 * max(abs(x[j]), 5)
        out[j] = 0.15 * cap if cap is not None else 0.1 * max(1.0, abs(x[j]))
    return out


def pt_scales(prob: PTProblem, x: np.ndarray, jtwj_diag: Optional[np.ndarray] = None) -> np.ndarray:
    nat = natural_scales(prob, x)
    if jtwj_diag is None:
        return nat
    sens = np.where(jtwj_diag > 0, 1 / np.sqrt(np.maximum(jtwj_diag, 1e-300)), nat)
    return np.maximum(np.maximum(nat, np.minimum(4 * nat, sens)), 1e-8)
