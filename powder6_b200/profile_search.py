"""Wyckoff search against a powder pattern with the cell and profile fixed.

With the cell and the peak profile held fixed, the calculated pattern of a
trial structure is y_calc = s * sum_k I_k col_k (+ the fixed background):
its reflection intensities I_k = mult_k |F_k|^2 times one banded profile
matrix whose columns carry the Lorentz-polarisation factor and the
Ka1/Ka2 peak shapes (js/profile.js:1013-1090, js/rietveld_core.js:855-917).
The scale s is the one that minimises the weighted chi^2 of each trial,
chi^2 = sum w y^2 - (sum w y Y)^2 / sum w Y^2.

``ProfileSearch`` runs the Wyckoff search (proposals, ladders, exchange and
penalty schedule of ``swarm_wyckoff``) with that chi^2 as its energy through
``p6_wy_profile_run``: per generation the search kernel evaluates every
replica's proposal and writes its intensity row, the contraction forms
Y = I . P for all replicas at once and reduces each replica's chi^2 at its
best scale in FP64, and an acceptance kernel applies the Metropolis test and
the ladder exchange.  The fitness is 1 - Rwp - penalty (Rwp on the
background-subtracted pattern).

The product runs with ``method``:
  * GRAM_FP64 -- no pattern at all: with the profile fixed, chi^2 at the
    best scale is sum w y^2 - (v . I)^2 / (I G I^T) with v = P (w y) and
    G = P W P^T fixed and banded, so the fused search kernel forms it from
    its FP64 intensities (``p6_wy_set_profile``) and every generation stays
    in one launch; exact in FP64;
  * SPLIT3_BF16 / SPLIT_BF16 -- the tensor cores (tcgen05, split-BF16, FP32
    accumulation) over each 256-point tile's band of reflections;
  * FP32_DENSE -- every reflection at every point on the CUDA cores in FP32,
    the dense render of the reference's `columns` and `targets` stages
    (js/pt_gpu.js:249-252);
  * FP32 -- the same CUDA-core product restricted to each tile's band.

``profile_problem`` builds the synthetic pattern of a Wyckoff problem's true
structure (Cu Ka1/Ka2, Caglioti widths, pseudo-Voigt peaks cut at a window of
FWHMs, a smooth known background, Poisson counts).
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Dict, Optional

import numpy as np

from . import _lib
from ._lib import check
from .contraction import FP32, FP32_DENSE, METHOD_NAMES, SPLIT3_BF16, SPLIT_BF16, ContractionSession
from .crystal import orth_matrix
from .swarm_wyckoff import (SW_DEFAULTS, WyckoffSession, build_ladders, initial_state, project_all,
                            reflection_intensities, schedule, weighted_assign, assignment_dims)
from .workloads import WyckoffProblem, mulberry32, wyckoff_problem

GRAM_FP64 = 4     # the fitted-scale chi^2 in Gram form inside the fused search (no contraction)
METHOD_NAMES = dict(METHOD_NAMES)
METHOD_NAMES[GRAM_FP64] = 'gram-fp64'

__all__ = ['ProfileProblem', 'profile_problem', 'profile_rwp', 'gram_operands', 'PatternGram', 'pattern_gram',
           'set_session_pattern', 'ProfileSearch', 'ProfileResult',
           'run_profile_search', 'SPLIT_BF16', 'SPLIT3_BF16', 'FP32', 'FP32_DENSE', 'GRAM_FP64', 'METHOD_NAMES']


@dataclass
class ProfileProblem:
    problem: WyckoffProblem
    tth: np.ndarray          # n_points, degrees
    tth_refl: np.ndarray     # per reflection (search order), Ka1 position
    fwhm: np.ndarray         # per reflection, degrees
    profile_t: np.ndarray    # n_points x n_refl float32: Lp (pV(Ka1) + ratio pV(Ka2)), unit height
    yobs: np.ndarray         # n_points float32: observed counts less the background
    w: np.ndarray            # n_points float32: 1 / max(counts, 1)
    background: np.ndarray   # n_points
    counts: np.ndarray       # n_points: the observed counts
    scale_true: float
    rwp_true: float          # Rwp of the true structure at its best scale (FP64)

    @property
    def n_points(self) -> int:
        return len(self.tth)

    @property
    def n_refl(self) -> int:
        return self.profile_t.shape[1]


def reflection_hkl(problem: WyckoffProblem) -> np.ndarray:
    pk = problem.refl.refl_pack[0::2].astype(np.int64)
    return np.stack([(pk & 0x3FF) - 512, ((pk >> 10) & 0x3FF) - 512, ((pk >> 20) & 0x3FF) - 512], 1)


def reflection_two_theta(problem: WyckoffProblem, wavelength: float) -> np.ndarray:
    """2-theta (degrees) of every reflection of the search from the cell metric."""
    A = orth_matrix(problem.cell).astype(np.float64).reshape(3, 3)
    gstar = np.linalg.inv(A.T @ A)
    h = reflection_hkl(problem).astype(np.float64)
    inv_d2 = np.einsum('ri,ij,rj->r', h, gstar, h)
    s = np.clip(wavelength * np.sqrt(inv_d2) / 2.0, 0.0, 1.0)
    return 2.0 * np.degrees(np.arcsin(s))


def pseudo_voigt(d: np.ndarray, fwhm: float, eta: float) -> np.ndarray:
    u = (d / fwhm) ** 2
    return eta / (1.0 + 4.0 * u) + (1.0 - eta) * np.exp(-4.0 * math.log(2.0) * u)


def profile_problem(problem: Optional[WyckoffProblem] = None, seed: int = 1, step: float = 0.01,
                    tth_lo: float = 5.0, wavelength: float = 1.5406, wavelength2: float = 1.5444,
                    ratio: float = 0.5, U: float = 0.004, V: float = -0.002, W: float = 0.003, eta: float = 0.5,
                    window: float = 20.0, peak_counts: float = 1.0e4, bkg0: float = 40.0,
                    bkg1: float = 60.0) -> ProfileProblem:
    """The pattern of ``problem``'s true structure (default: the Pnma
    PbSO4-like problem of ``wyckoff_problem``): points from ``tth_lo`` to
    2 degrees past the last reflection at ``step``; each reflection a
    pseudo-Voigt of Caglioti width sqrt(U tan^2 th + V tan th + W) at Ka1
    and, ``ratio`` times as high, at Ka2, cut at +/- ``window`` FWHM and
    multiplied by Lp = (1 + cos^2 2th) / (sin^2 th cos th); the scale puts
    the tallest net peak at ``peak_counts``; background bkg0 + bkg1 exp(-2th
    / 25); Poisson counts; weights 1 / max(counts, 1)."""
    prob = problem if problem is not None else wyckoff_problem(seed=1)
    if prob.true_coords is None:
        raise ValueError('the problem has no true structure to make a pattern from')
    rng = np.random.default_rng(seed)
    t1 = reflection_two_theta(prob, wavelength)
    s2 = np.clip(np.sin(np.radians(t1 / 2.0)) * wavelength2 / wavelength, 0.0, 1.0)
    t2 = 2.0 * np.degrees(np.arcsin(s2))
    th = np.radians(t1 / 2.0)
    fw = np.sqrt(np.maximum(U * np.tan(th) ** 2 + V * np.tan(th) + W, 1e-6))
    lp = (1.0 + np.cos(2 * th) ** 2) / (np.sin(th) ** 2 * np.cos(th))
    tth_hi = float(np.max(t2)) + 2.0
    tth = tth_lo + step * np.arange(int(math.floor((tth_hi - tth_lo) / step)) + 1)
    K = len(t1)
    pt = np.zeros((len(tth), K), dtype=np.float64)
    for k in range(K):
        for centre, hgt in ((t1[k], 1.0), (t2[k], ratio)):
            half = window * fw[k]
            lo = int(np.searchsorted(tth, centre - half, 'left'))
            hi = int(np.searchsorted(tth, centre + half, 'right'))
            if hi > lo:
                pt[lo:hi, k] += hgt * lp[k] * pseudo_voigt(tth[lo:hi] - centre, fw[k], eta)
    I = reflection_intensities(prob, prob.true_coords, 0)
    net = pt @ I
    scale = peak_counts / float(np.max(net))
    bkg = bkg0 + bkg1 * np.exp(-tth / 25.0)
    counts = rng.poisson(scale * net + bkg).astype(np.float64)
    w = 1.0 / np.maximum(counts, 1.0)
    yobs = counts - bkg
    pp = ProfileProblem(prob, tth, t1, fw, pt.astype(np.float32), yobs.astype(np.float32), w.astype(np.float32),
                        bkg, counts, scale, 0.0)
    pp.rwp_true = float(profile_rwp(pp, I[None, :])[0])
    return pp


def profile_rwp(pp: ProfileProblem, intensities: np.ndarray, n_active_points: Optional[int] = None) -> np.ndarray:
    """Rwp at the best scale of each row of ``intensities`` (FP64): the
    product's re-score of a search's winners."""
    n = pp.n_points if n_active_points is None else int(n_active_points)
    I = np.atleast_2d(np.asarray(intensities, dtype=np.float64))
    Y = I @ pp.profile_t[:n].astype(np.float64).T
    w = np.maximum(pp.w[:n].astype(np.float64), 0.0)
    y = pp.yobs[:n].astype(np.float64)
    syy = float(np.sum(w * y * y))
    a = Y @ (w * y)
    b = (Y * Y) @ w
    chi = np.where((a > 0) & (b > 0), syy - a * a / np.where(b > 0, b, 1.0), syy)
    return np.sqrt(np.maximum(chi, 0.0) / syy)


def gram_operands(pp: ProfileProblem, n_active_points: Optional[int] = None):
    """v = P (w y) per reflection, the upper band of G = P W P^T by diagonal
    (band[d, k] = G[k, k + d]), its width and sum w y^2, in FP64, over the
    first ``n_active_points`` points: the fixed profile's whole contribution
    to chi^2 at the best scale."""
    n = pp.n_points if n_active_points is None else int(n_active_points)
    PT = pp.profile_t[:n].astype(np.float64)
    w = np.maximum(pp.w[:n].astype(np.float64), 0.0)
    y = pp.yobs[:n].astype(np.float64)
    v = PT.T @ (w * y)
    G = PT.T @ (w[:, None] * PT)
    K = G.shape[0]
    nz = np.abs(G) > 0
    bw = 0
    for k in range(K):
        cols = np.flatnonzero(nz[k, k:])
        if len(cols):
            bw = max(bw, int(cols[-1]))
    band = np.zeros((bw + 1, K))
    for d in range(bw + 1):
        band[d, :K - d] = np.diagonal(G, d)
    return v, band, bw, float(np.sum(w * y * y))


@dataclass
class PatternGram:
    """A pattern reduced to what the Gram-form fitness reads (``gram_operands``),
    built without the dense profile matrix."""
    v: np.ndarray
    band: np.ndarray
    bw: int
    syy: float
    n_points: int
    rwp_true: float


def pattern_gram(problem: WyckoffProblem, n_points: Optional[int] = None, seed: int = 1, step: float = 0.01,
                 wavelength: float = 1.5406,
                 wavelength2: float = 1.5444, ratio: float = 0.5, U: float = 0.004, V: float = -0.002,
                 W: float = 0.003, eta: float = 0.5, window: float = 20.0, peak_counts: float = 1.0e4,
                 bkg0: float = 40.0, bkg1: float = 60.0, tth_lo: float = 5.0) -> PatternGram:
    """The pattern of ``profile_problem`` for ``problem``'s true structure,
    from ``tth_lo`` to 2 degrees past the last reflection at ``step`` (or
    ``n_points`` evenly spaced points), kept as a sparse profile matrix: the
    Gram operands v = P (w y) and the band of G = P W P^T, and the true
    structure's Rwp (FP64).  The Gram form costs n_refl x (bw + 1) FMAs per
    trial, so it suits patterns whose reflections overlap little."""
    from scipy import sparse
    if problem.true_coords is None:
        raise ValueError('the problem has no true structure to make a pattern from')
    rng = np.random.default_rng(seed)
    t1 = reflection_two_theta(problem, wavelength)
    t2 = 2.0 * np.degrees(np.arcsin(np.clip(np.sin(np.radians(t1 / 2.0)) * wavelength2 / wavelength, 0.0, 1.0)))
    th = np.radians(t1 / 2.0)
    fw = np.sqrt(np.maximum(U * np.tan(th) ** 2 + V * np.tan(th) + W, 1e-6))
    lp = (1.0 + np.cos(2 * th) ** 2) / (np.sin(th) ** 2 * np.cos(th))
    tth_hi = float(np.max(t2)) + 2.0
    if n_points is None:
        tth = tth_lo + step * np.arange(int(math.floor((tth_hi - tth_lo) / step)) + 1)
    else:
        tth = np.linspace(tth_lo, tth_hi, int(n_points))
    rows, cols, vals = [], [], []
    for k in range(len(t1)):
        lo = int(np.searchsorted(tth, min(t1[k], t2[k]) - window * fw[k], 'left'))
        hi = int(np.searchsorted(tth, max(t1[k], t2[k]) + window * fw[k], 'right'))
        if hi <= lo:
            continue
        x = tth[lo:hi]
        col = np.zeros(hi - lo)
        for centre, hgt in ((t1[k], 1.0), (t2[k], ratio)):
            m = np.abs(x - centre) <= window * fw[k]
            col[m] += hgt * lp[k] * pseudo_voigt(x[m] - centre, fw[k], eta)
        nz = col != 0
        rows.append(np.arange(lo, hi)[nz])
        cols.append(np.full(int(nz.sum()), k))
        vals.append(col[nz])
    K = len(t1)
    P = sparse.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(len(tth), K))
    I = reflection_intensities(problem, problem.true_coords, 0)
    net = P @ I
    scale = peak_counts / float(np.max(net))
    bkg = bkg0 + bkg1 * np.exp(-tth / 25.0)
    counts = rng.poisson(scale * net + bkg).astype(np.float64)
    w = 1.0 / np.maximum(counts, 1.0)
    y = counts - bkg
    v = P.T @ (w * y)
    G = (P.T @ sparse.diags(w) @ P).tocoo()
    up = G.col >= G.row
    d = G.col[up] - G.row[up]
    bw = int(d.max()) if d.size else 0
    band = np.zeros((bw + 1, K))
    band[d, G.row[up]] = G.data[up]
    syy = float(np.sum(w * y * y))
    a, b = float(I @ v), float(np.sum((P @ I) ** 2 * w))
    chi = syy - a * a / b if a > 0 and b > 0 else syy
    return PatternGram(np.asarray(v, dtype=np.float64), band, bw, syy, len(tth), float(np.sqrt(max(chi, 0.0) / syy)))


def set_session_pattern(session: WyckoffSession, pg: Optional[PatternGram]):
    """The Gram-form profile fitness for a search session (``p6_wy_set_profile``);
    None returns it to the grouped-intensity fitness."""
    if pg is None:
        check(session.lib.p6_wy_set_profile(session.h, None, None, 0, 0.0))
        return
    v = np.ascontiguousarray(pg.v, dtype=np.float64)
    band = np.ascontiguousarray(pg.band, dtype=np.float64)
    session._pattern_keep = (v, band)
    check(session.lib.p6_wy_set_profile(session.h, v.ctypes.data, band.ctypes.data, int(pg.bw), float(pg.syy)))


@dataclass
class ProfileResult:
    best_rwp: float
    best_pen: float
    best_coords: np.ndarray
    best_assignment: int
    generations: int
    trials: int
    device_ms: float
    wall_s: float
    accept_rate: float
    method: str
    seed: int
    time_to_target: Optional[float] = None
    generations_to_target: Optional[int] = None
    cpu_check: Dict[str, float] = field(default_factory=dict)


class ProfileSearch:
    """A Wyckoff search session and a contraction session over the same
    reflections (``p6_wy_profile_run``)."""

    def __init__(self, pp: ProfileProblem, num_particles: int = 4096, run_key: int = 1,
                 cos_mode: Optional[int] = None, device: int = 0, settings: Optional[dict] = None):
        self.pp = pp
        self.lib = _lib.load()
        self.settings = dict(SW_DEFAULTS)
        self.settings.update(settings or {})
        self.wy = WyckoffSession(pp.problem, num_particles, run_key=run_key, cos_mode=cos_mode, device=device,
                                 settings=settings, incremental=0)
        self.ct = ContractionSession(_ContractionInput(pp), max_replicas=num_particles, device=device)
        self.ct.set_fitted(True)
        self.num_particles = self.wy.num_particles
        self.assign_of = np.zeros(self.num_particles, dtype=np.uint32)
        self.n_gen = 0
        self._gram = None
        self._gram_on = False

    def set_gram(self, on: bool):
        """The search kernel's own fitness: the Gram form of the profile chi^2
        (on) or the grouped intensities (off)."""
        if on and not self._gram_on:
            if self._gram is None:
                v, band, bw, syy = gram_operands(self.pp)
                self._gram = (np.ascontiguousarray(v), np.ascontiguousarray(band), bw, syy)
            v, band, bw, syy = self._gram
            check(self.lib.p6_wy_set_profile(self.wy.h, v.ctypes.data, band.ctypes.data, int(bw), float(syy)))
        elif not on and self._gram_on:
            check(self.lib.p6_wy_set_profile(self.wy.h, None, None, 0, 0.0))
        self._gram_on = bool(on)

    def close(self):
        self.wy.close()
        self.ct.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def start(self, generations: int, seed: int, assignment_ids=None, method: int = SPLIT_BF16):
        """Random start (``prepare``), then the first evaluation of the
        current structures."""
        self.prepare(generations, seed, assignment_ids)
        self.run(0, 0, method, init=True)

    def prepare(self, generations: int, seed: int, assignment_ids=None):
        """The host side of a random start: particles shared over the
        assignments by free parameters, ladders, the penalty schedule, random
        coordinates and states uploaded."""
        d = self.settings
        prob = self.pp.problem
        n = self.num_particles
        nA = len(prob.assignments)
        ids = list(range(nA)) if assignment_ids is None else [int(a) for a in assignment_ids]
        self.assign_of = weighted_assign(ids, n, int(d['minParticlesPerAssignment']), assignment_dims(prob))
        self.wy.set_assign(self.assign_of)
        ladders, temps = build_ladders(self.assign_of, int(d['rungs']), d['tempCold'], d['tempHot'])
        self.wy.set_ladders(ladders, max(2, int(d['rungs'])))
        groups, pen = schedule(generations, prob.refl.n_groups, d)
        groups[:] = prob.refl.n_groups     # the pattern needs every reflection: no resolution ramp
        self.wy.set_schedule(groups, pen)
        self.pen0 = float(pen[0])
        self.pen_final = float(pen[-1])
        self.n_gen = generations
        rnd = mulberry32(seed)
        cpp = self.wy.coords_per_particle
        pos = project_all(prob, np.array([rnd() for _ in range(n * cpp)], dtype=np.float32), self.assign_of)
        self.wy.sync_state(pos, initial_state(n, temps, rnd, d))

    def run(self, gen0: int, n_gen: int, method: int = SPLIT_BF16, swap_every: Optional[int] = None,
            init: bool = False, n_active_points: int = 0):
        se = int(self.settings['swapEvery']) if swap_every is None else int(swap_every)
        if method == GRAM_FP64:
            # the fused search with the Gram-form fitness: all generations in one launch
            self.set_gram(True)
            if init:
                self.wy.set_params(self.pp.problem.refl.n_groups, self.pen0)
                self.wy.dispatch(None, mcmc=False)
            if n_gen > 0:
                self.wy.run(int(gen0), int(n_gen), se, reeval_first=False)
            return
        self.set_gram(False)
        check(self.lib.p6_wy_profile_run(self.wy.h, self.ct.h, int(method), int(gen0), int(n_gen), se,
                                         1 if init else 0, int(n_active_points)))

    def synchronize(self, timeout: float = 600.0):
        self.wy.synchronize(timeout)

    def last_ms(self) -> float:
        return self.wy.last_kernel_ms()

    def best(self):
        """(best Rwp over the replicas, its penalty, coordinates, assignment)."""
        _, bestpos, st = self.wy.read_state()
        ok = st['best_fit'] > -1e29
        if not np.any(ok):
            return 1.0, 0.0, None, 0
        i = int(np.flatnonzero(ok)[np.argmax(st['best_cc'][ok])])
        cpp = self.wy.coords_per_particle
        return (1.0 - float(st['best_cc'][i]), float(st['best_pen'][i]), bestpos[i * cpp:(i + 1) * cpp].copy(),
                int(self.assign_of[i]))


class _ContractionInput:
    """The fields ContractionSession reads, from a ProfileProblem."""

    def __init__(self, pp: ProfileProblem):
        self.profile_t = pp.profile_t
        self.yobs = pp.yobs
        self.w = pp.w
        self.intensities = np.zeros((1, pp.n_refl), dtype=np.float32)


def run_profile_search(pp: ProfileProblem, num_particles: int = 4096, generations: int = 2000, seed: int = 1,
                       method: int = SPLIT_BF16, chunk: int = 100, target_rwp: Optional[float] = None,
                       search: Optional[ProfileSearch] = None, settings: Optional[dict] = None,
                       stop_at_target: bool = False) -> ProfileResult:
    """One search from a random start, in chunks of ``chunk`` generations
    (the best is read between chunks).  With ``target_rwp``,
    ``time_to_target`` is the wall time from the first evaluation of the
    random start (the host's drawing and upload of it excluded) to the
    first chunk boundary at which the best Rwp is at or below it;
    ``stop_at_target`` ends the search there.
    The winner is re-scored in FP64 on the host (``cpu_check``)."""
    own = search is None
    ps = search or ProfileSearch(pp, num_particles, run_key=seed, settings=settings)
    try:
        ps.prepare(generations, seed)
        ps.synchronize()
        t0 = time.perf_counter()
        ps.run(0, 0, method, init=True)
        ps.synchronize()
        dev_ms = ps.last_ms()
        hit, hit_gen = None, None
        g0 = 0
        while g0 < generations:
            ng = min(chunk, generations - g0)
            ps.run(g0, ng, method)
            ps.synchronize()
            dev_ms += ps.last_ms()
            g0 += ng
            if target_rwp is not None and hit is None:
                _, _, stc = ps.wy.read_state()
                ok = stc['best_fit'] > -1e29
                if np.any(ok) and 1.0 - float(np.max(stc['best_cc'][ok])) <= target_rwp:
                    hit, hit_gen = time.perf_counter() - t0, g0
                    if stop_at_target:
                        break
        wall = time.perf_counter() - t0
        rwp, pen, coords, A = ps.best()
        _, _, st = ps.wy.read_state()
        acc = float(np.sum(st['accepted'])) / max(1, ps.num_particles * g0)
        cpu = {}
        if coords is not None:
            I = reflection_intensities(pp.problem, coords, A)
            r64 = float(profile_rwp(pp, I[None, :])[0])
            cpu = {'rwp_fp64': r64, 'rwp_device': rwp, 'delta': abs(r64 - rwp)}
        return ProfileResult(rwp, pen, coords, A, g0, ps.num_particles * g0, dev_ms, wall, acc,
                             METHOD_NAMES[method], seed, hit, hit_gen, cpu)
    finally:
        if own:
            ps.close()


def main(argv=None):
    """python -m powder6_b200.profile_search: a short fixed-profile search of
    the PbSO4-like pattern with each method named, or (--contract-evals)
    only the fitted-scale contraction of random intensity rows; one JSON
    line per method."""
    import argparse
    import json
    names = {v: k for k, v in METHOD_NAMES.items()}
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument('--replicas', type=int, default=4096)
    ap.add_argument('--generations', type=int, default=10)
    ap.add_argument('--methods', default='split3-bf16,fp32-dense', help=', '.join(names))
    ap.add_argument('--seed', type=int, default=3)
    ap.add_argument('--contract-evals', type=int, default=0,
                    help='evaluate the contraction this many times on random rows instead of searching')
    a = ap.parse_args(argv)
    methods = [names[m] for m in a.methods.split(',') if m]
    pp = profile_problem()
    if a.contract_evals > 0:
        I = np.random.default_rng(a.seed).lognormal(0.0, 1.5, (a.replicas, pp.n_refl)).astype(np.float32)
        with ContractionSession(_ContractionInput(pp), max_replicas=a.replicas) as s:
            s.set_fitted(True)
            s.set_intensities(I)
            for m in methods:
                for _ in range(a.contract_evals):
                    s.evaluate(m)
                s.synchronize()
                print(json.dumps({'method': METHOD_NAMES[m], 'ms_per_evaluation': s.last_ms()}), flush=True)
        return
    with ProfileSearch(pp, a.replicas, run_key=a.seed) as ps:
        for m in methods:
            ps.start(max(a.generations, 2), seed=a.seed, method=m)
            ps.run(0, a.generations, m)
            ps.synchronize()
            rwp, _, _, _ = ps.best()
            print(json.dumps({'method': METHOD_NAMES[m], 'generations': a.generations, 'best_rwp': rwp,
                              'rwp_true': pp.rwp_true, 'ms_last_run': ps.last_ms()}), flush=True)


if __name__ == '__main__':
    main()
