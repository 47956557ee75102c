"""The Wyckoff worker's message protocol on the host, over the CUDA search.

The reference runs the Wyckoff search in a Web Worker that takes one job
message and answers with a stream of messages (js/wyckoff_worker.js:1782-1861;
the page's side is js/rietveld/rv_solve.js:774-803):

* in: ``{type: 'wyckoff-search', cell, symops, wyckoffTable,
  targetComposition, wyckoffZ, hklList, swarmParticles, swarmIterations,
  swarmRestarts, seed, minContact, distanceConstraints, polyProb, ...}`` and
  ``{type: 'cancel-wyckoff'}``, which arrives while a search runs and asks
  for the best structure so far;
* out: ``wy-start``, ``wy-info``, ``wy-log``, ``wy-progress`` (the fields of
  js/wyckoff_worker.js:1545-1556), ``wy-partial`` (one per finished Z),
  ``wy-refining``, ``wy-structure`` (the result, :1825-1856) and ``wy-error``
  (every failure, and any message type other than the two above, :1789-1797).

``WyckoffWorker`` keeps that schema.  ``post`` stands for the Worker's
``postMessage`` (a Python callable here; an N-API host would forward the
dicts as JS objects).  The search itself is ``swarm_wyckoff.run_wyckoff_waves``
on the device; a cancel is honoured between kernel launches, as the
reference's ``shouldStop`` is between dispatches.

What is built here from the job, in the reference's terms:

* the space group from ``symops`` (``{r, t_num, t_den}`` or ``xyz`` strings)
  and the Wyckoff positions from ``wyckoffTable`` (letter, multiplicity,
  ``special_op``), as the sg/all.json settings carry them;
* the observations from ``hklList`` by normaliseObservations' routes
  (js/observations.js:161-212): |F|^2 = I / (m Lp) with the row's own Lp when
  every row has m and Lp, else Lp from 2-theta and the polarisation ratio K
  (js/crystal.js:438-492), sigma scaled with its value; negative and
  non-finite intensities are dropped and counted (js/wyckoff_worker.js:164-212);
* the cell contents from ``targetComposition`` x Z; Z from ``wyckoffZ`` or,
  when absent, every Z whose density lies in [densityMin, densityMax], most
  plausible first, at most ``maxZSearches`` of them;
* the assignments from ``wyckoff_assign.enumerate_assignments`` with the
  normaliser deduplication.
"""
from __future__ import annotations

import math
import re
import threading
import traceback
from fractions import Fraction
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from .symmetry import TDEN, SpaceGroup, SymOp, _parse_triplet, build_wyckoff

DEFAULT_PARTICLES = 4096
DEFAULT_GENERATIONS = 1000
DEFAULT_RESTARTS = 1
DEFAULT_MAX_Z = 3
DEFAULT_DENSITY = (1.0, 10.0)      # g/cm^3, the window an automatic Z is drawn from
PROGRESS_CHUNKS = 10               # progress messages per restart

# Standard atomic weights (IUPAC, abridged) of the elements the scattering table carries.
ATOMIC_MASS = {'H': 1.008, 'C': 12.011, 'N': 14.007, 'O': 15.999, 'Na': 22.990, 'S': 32.06, 'Cl': 35.45,
               'Ti': 47.867, 'Fe': 55.845, 'Pb': 207.2}
AVOGADRO_CM3 = 1.66053907  # g/cm^3 per (atomic mass unit / A^3)


class JobError(ValueError):
    """A job the search cannot run; its message is posted as wy-error."""


class CombinatorialError(JobError):
    """No assignment exists for one Z: it rules out that Z only."""


# ---------------------------------------------------------------------------
# Job -> problem
# ---------------------------------------------------------------------------

def parse_formula(formula: str) -> List[Tuple[str, int]]:
    """'PbSO4', 'C10N6S', 'Ca(OH)2' -> [(element, count)] in first-seen order."""
    tokens = re.findall(r'([A-Z][a-z]?|\(|\)|\d+)', formula.replace(' ', ''))
    if ''.join(tokens) != formula.replace(' ', ''):
        raise JobError(f'Cannot read the composition "{formula}".')
    stack: List[Dict[str, int]] = [{}]
    order: List[str] = []
    i = 0
    while i < len(tokens):
        t = tokens[i]
        n = int(tokens[i + 1]) if i + 1 < len(tokens) and tokens[i + 1].isdigit() else 1
        step = 2 if i + 1 < len(tokens) and tokens[i + 1].isdigit() else 1
        if t == '(':
            stack.append({})
            i += 1
            continue
        if t == ')':
            if len(stack) < 2:
                raise JobError(f'Unbalanced parentheses in "{formula}".')
            inner = stack.pop()
            for el, c in inner.items():
                stack[-1][el] = stack[-1].get(el, 0) + c * n
            i += step
            continue
        if t.isdigit():
            raise JobError(f'Cannot read the composition "{formula}".')
        if t not in order:
            order.append(t)
        stack[-1][t] = stack[-1].get(t, 0) + n
        i += step
    if len(stack) != 1 or not stack[0]:
        raise JobError(f'Cannot read the composition "{formula}".')
    return [(el, stack[0][el]) for el in order if stack[0].get(el, 0) > 0]


def _op_from_entry(o) -> SymOp:
    if isinstance(o, str) or (isinstance(o, dict) and 'r' not in o):
        xyz = o if isinstance(o, str) else o.get('xyz')
        if not xyz:
            raise JobError('A symmetry operator carries neither a matrix nor an x,y,z form.')
        comps = _parse_triplet(xyz)
        r = tuple(int(c) for comp in comps for c in comp[0])
        t = tuple(int((comp[1] * TDEN) % TDEN) for comp in comps)
        if any((comp[1] * TDEN).denominator != 1 for comp in comps):
            raise JobError(f'Operator "{xyz}" has a translation that is not a multiple of 1/{TDEN}.')
        return SymOp(r, t)
    r = tuple(int(round(v)) for v in o['r'])
    if 't_num' in o and 't_den' in o:
        num = [Fraction(int(v), int(o['t_den'])) for v in o['t_num']]
    else:
        num = [Fraction(float(v)).limit_denominator(TDEN) for v in o['t']]
    t = tuple(int((v * TDEN) % TDEN) for v in num)
    return SymOp(r, t)


def group_from_job(symops: Sequence, wyckoff_table: Sequence[dict], symbol: str = '') -> SpaceGroup:
    """The job's operators and Wyckoff table as a SpaceGroup (site projectors,
    coset operators and stabiliser orders are rebuilt from the operators)."""
    ops = [_op_from_entry(o) for o in symops]
    if len({(o.r, o.t) for o in ops}) != len(ops):
        raise JobError('The symmetry operators contain duplicates.')
    g = SpaceGroup(0, symbol, '', '', ops)
    g.wyckoff = []
    for w in wyckoff_table:
        trip = w.get('special_op') or w.get('xyz')
        if not trip:
            raise JobError(f'Wyckoff position {w.get("letter", "?")} carries no coordinate triplet.')
        try:
            g.wyckoff.append(build_wyckoff(ops, str(w['letter']), int(w['multiplicity']), trip))
        except ValueError as e:
            raise JobError(f'The Wyckoff table does not match the operators: {e}') from None
    g.site_symmetry = {str(w['letter']): str(w.get('site_symmetry', '')) for w in wyckoff_table}
    return g


def polarisation_k(job: dict) -> float:
    """sharkoPolarizationK (js/crystal.js:438-458) of the job's descriptor."""
    if job.get('radiation') == 'neutron':
        return 0.0
    pol = job.get('polarization', job.get('monochromatorTth'))
    if isinstance(pol, (int, float)) and not isinstance(pol, bool):
        return math.cos(math.radians(pol)) ** 2 if 0 < pol < 180 else 1.0
    if isinstance(pol, dict):
        if isinstance(pol.get('K'), (int, float)) and pol['K'] >= 0:
            return float(pol['K'])
        mode = str(pol.get('mode', 'monochromator')).lower()
        if mode == 'none':
            return 0.0
        if mode == 'synchrotron':
            f = pol.get('polFrac')
            if not isinstance(f, (int, float)) or f >= 1:
                return 0.0
            return 1e6 if f <= 1e-6 else (1 - f) / f
        m = pol.get('monoTth')
        return math.cos(math.radians(m)) ** 2 if isinstance(m, (int, float)) and 0 < m < 180 else 1.0
    return 1.0


def lorentz_polarisation(tth: float, k: float) -> float:
    """sharkoLorentzPolarization (js/crystal.js:465-492): 1 where the geometry is degenerate."""
    if not (isinstance(tth, (int, float)) and 0 < tth < 180):
        return 1.0
    th = math.radians(0.5 * tth)
    s, c = math.sin(th), math.cos(th)
    if s < 1e-6 or c < 1e-6:
        return 1.0
    return (1.0 / (s * s * c)) * (1 + k * math.cos(math.radians(tth)) ** 2) / (1 + k)


def _num(v) -> float:
    try:
        x = float(v)
    except (TypeError, ValueError):
        return float('nan')
    return x


def observation_rows(job: dict) -> Tuple[List[dict], List[str]]:
    """hklList -> rows {h, k, l, mult, Fo2, sigma, d, tth} and the warnings to log."""
    lam = _num(job.get('wavelength'))
    apply_lp = job.get('applyLP', True) is not False
    K = polarisation_k(job)
    src, negative, non_finite = [], 0, 0
    for p in job.get('hklList') or []:
        if not p:
            continue
        I = _num(p.get('intensity'))
        h, k, l = p.get('h_orig', p.get('h')), p.get('k_orig', p.get('k')), p.get('l_orig', p.get('l'))
        if not math.isfinite(I):
            non_finite += 1
            continue
        if I < 0:
            negative += 1
            continue
        if not all(isinstance(v, (int, float)) and math.isfinite(v) for v in (h, k, l)):
            continue
        h, k, l = int(h), int(k), int(l)
        if h == 0 and k == 0 and l == 0:
            continue
        if max(abs(h), abs(k), abs(l)) > 511:
            continue
        d, tth = _num(p.get('d')), _num(p.get('tth', p.get('twoTheta')))
        if not math.isfinite(d) and math.isfinite(tth) and lam > 0:
            s = math.sin(math.radians(0.5 * tth))
            d = lam / (2 * s) if s > 1e-9 else float('nan')
        if not math.isfinite(tth) and math.isfinite(d) and lam > 0 and lam / (2 * d) < 1:
            tth = 2 * math.degrees(math.asin(lam / (2 * d)))
        src.append({'h': h, 'k': k, 'l': l, 'I': I, 'm': p.get('multiplicity'), 'lp': _num(p.get('lp')),
                    'sigma': _num(p.get('sigma')), 'd': d, 'tth': tth})
    warnings = []
    if negative or non_finite:
        warnings.append(f'{negative} reflection(s) with a NEGATIVE extracted intensity'
                        + (f' and {non_finite} non-numeric' if non_finite else '')
                        + ' were dropped from the search.')
    if not src:
        raise JobError('The job carries no usable intensity.')
    if not all(isinstance(r['m'], (int, float)) and r['m'] > 0 for r in src):
        raise JobError('The reflection list does not state the powder multiplicity of every reflection.')
    have_lp = all(math.isfinite(r['lp']) and r['lp'] > 0 for r in src)
    rows = []
    for r in src:
        if not (r['d'] > 0):
            continue
        if not apply_lp:
            lp = 1.0
        elif have_lp:
            lp = r['lp']
        elif math.isfinite(r['tth']):
            lp = lorentz_polarisation(r['tth'], K)
        else:
            raise JobError('Neither Lp nor 2-theta (or d with a wavelength) is given, so the '
                           'Lorentz-polarisation factor cannot be removed.')
        f = 1.0 / (int(r['m']) * lp)
        sig = r['sigma'] * f if math.isfinite(r['sigma']) and r['sigma'] > 0 else None
        rows.append({'h': r['h'], 'k': r['k'], 'l': r['l'], 'mult': int(r['m']), 'Fo2': r['I'] * f,
                     'sigma': sig, 'd': r['d'], 'tth': r['tth']})
    if not rows:
        raise JobError('No reflection has a usable d-spacing.')
    return rows, warnings


def cell_volume(cell: dict) -> float:
    al, be, ga = (math.radians(float(cell.get(k, 90.0))) for k in ('alpha', 'beta', 'gamma'))
    return float(cell['a']) * float(cell['b']) * float(cell['c']) * math.sqrt(
        max(0.0, 1 - math.cos(al) ** 2 - math.cos(be) ** 2 - math.cos(ga) ** 2
            + 2 * math.cos(al) * math.cos(be) * math.cos(ga)))


def z_plan(job: dict, formula: Sequence[Tuple[str, int]], group: SpaceGroup) -> Tuple[List[int], bool]:
    """The Z values to try and whether Z was chosen automatically."""
    z = job.get('wyckoffZ')
    if isinstance(z, (int, float)) and not isinstance(z, bool) and z > 0:
        if int(z) != z:
            raise JobError(f'Z = {z} is not a whole number.')
        return [int(z)], False
    mass = 0.0
    for el, n in formula:
        if el not in ATOMIC_MASS:
            raise JobError(f'No atomic mass for {el}: give Z explicitly.')
        mass += ATOMIC_MASS[el] * n
    lo = _num(job.get('densityMin'))
    hi = _num(job.get('densityMax'))
    lo = lo if math.isfinite(lo) and lo > 0 else DEFAULT_DENSITY[0]
    hi = hi if math.isfinite(hi) and hi > lo else max(lo * 2, DEFAULT_DENSITY[1])
    vol = cell_volume(job['cell'])
    zmax = 4 * len(group.ops)
    cands = []
    for Z in range(1, zmax + 1):
        rho = Z * mass * AVOGADRO_CM3 / vol
        if lo <= rho <= hi:
            cands.append((abs(math.log(rho / math.sqrt(lo * hi))), Z))
    if not cands:
        raise JobError(f'No Z gives a density between {lo:g} and {hi:g} g/cm^3 for this cell.')
    cap = job.get('maxZSearches')
    cap = int(cap) if isinstance(cap, (int, float)) and cap >= 1 else DEFAULT_MAX_Z
    return [Z for _, Z in sorted(cands)[:cap]], True


def problem_for_z(job: dict, group: SpaceGroup, formula: Sequence[Tuple[str, int]], Z: int,
                  rows: Sequence[dict]):
    """(problem, assignment records) for one Z; CombinatorialError when no assignment exists."""
    from .workloads import build_problem, load_form_factor_table
    from .wyckoff_assign import assignment_labels, dedupe_equivalent_assignments, enumerate_assignments
    ff = load_form_factor_table()
    demand = [{'element': el, 'count': n * Z, 'z': ff[el]['Z'] if el in ff else 1} for el, n in formula]
    opts = {}
    if isinstance(job.get('wyckoffMaxSites'), (int, float)) and job['wyckoffMaxSites'] > 0:
        opts['maxSites'] = int(job['wyckoffMaxSites'])
    if isinstance(job.get('wyckoffMaxRepeat'), (int, float)) and job['wyckoffMaxRepeat'] > 0:
        opts['maxRepeat'] = int(job['wyckoffMaxRepeat'])
    en = enumerate_assignments(group, demand, opts)
    if en.get('error'):
        raise CombinatorialError(en['error'])
    found = en['assignments']
    if not found:
        raise CombinatorialError('No Wyckoff assignment matches this composition.')
    found = dedupe_equivalent_assignments(found, group)['assignments']
    labels = [assignment_labels(group, a) for a in found]
    prob = build_problem(group, job['cell'], demand, labels, rows, job.get('distanceConstraints') or [],
                         job.get('minContact'), overall_b=_num(job.get('overallB')) if
                         math.isfinite(_num(job.get('overallB'))) else 0.0)
    return prob, labels


def site_records(problem, A: int, coords: np.ndarray) -> List[dict]:
    """The sites of assignment A at ``coords`` as the page reads them."""
    sym = getattr(problem.group, 'site_symmetry', {})
    out = []
    for si, s in enumerate(problem.assignments[A].sites):
        x, y, z = (v % 1.0 for v in s.w.project(*[float(v) for v in coords[3 * si:3 * si + 3]]))
        out.append({'element': s.element, 'wyckoff': f'{s.w.multiplicity}{s.w.letter}',
                    'multiplicity': s.w.multiplicity, 'siteSymmetry': sym.get(s.w.letter, ''),
                    'x': x, 'y': y, 'z': z})
    return out


# ---------------------------------------------------------------------------
# The worker
# ---------------------------------------------------------------------------

class WyckoffWorker:
    """One Wyckoff worker: ``on_message`` takes the reference's messages and
    ``post`` receives the answers.  A search runs on a thread of its own
    (``threaded``) so that ``cancel-wyckoff`` can arrive while it runs;
    ``join`` waits for it.  ``search`` defaults to the device search
    (``swarm_wyckoff.run_wyckoff_waves``) and takes the same arguments."""

    def __init__(self, post: Callable[[dict], None], search: Optional[Callable] = None, threaded: bool = True,
                 device: int = 0):
        self.post = post
        self.search = search
        self.threaded = threaded
        self.device = device
        self._stop = threading.Event()
        self._thread: Optional[threading.Thread] = None

    # The reference answers every message except a cancel (js/wyckoff_worker.js:1785-1797).
    def on_message(self, msg: Optional[dict]):
        job = msg or {}
        kind = job.get('type')
        if kind == 'cancel-wyckoff':
            self._stop.set()
            return
        if kind != 'wyckoff-search':
            self.post({'type': 'wy-error', 'message': f'The Wyckoff worker does not handle job type "{kind}".'})
            return
        if self._thread is not None and self._thread.is_alive():
            self.post({'type': 'wy-error', 'message': 'A Wyckoff search is already running in this worker.'})
            return
        self._stop.clear()
        if self.threaded:
            self._thread = threading.Thread(target=self._run_job, args=(job,), daemon=True)
            self._thread.start()
        else:
            self._run_job(job)

    def join(self, timeout: Optional[float] = None) -> bool:
        if self._thread is not None:
            self._thread.join(timeout)
            return not self._thread.is_alive()
        return True

    def stop_requested(self) -> bool:
        return self._stop.is_set()

    def _log(self, text: str):
        self.post({'type': 'wy-log', 'message': str(text)})

    def _run_job(self, job: dict):
        try:
            self._search_job(job)
        except JobError as e:
            self.post({'type': 'wy-error', 'message': str(e)})
        except Exception as e:   # every failure is answered, never a silent worker
            self._log(traceback.format_exc())
            self.post({'type': 'wy-error', 'message': str(e) or e.__class__.__name__})

    def _search_job(self, job: dict):
        symops = job.get('symops') or []
        if not symops:
            raise JobError('No symmetry operators for the chosen setting.')
        if not job.get('targetComposition'):
            raise JobError('A target composition is required for a Wyckoff search.')
        if not job.get('wyckoffTable'):
            raise JobError('This setting carries no Wyckoff table.')
        if not isinstance(job.get('cell'), dict) or not all(k in job['cell'] for k in ('a', 'b', 'c')):
            raise JobError('The job carries no unit cell.')
        self.post({'type': 'wy-start', 'message': 'Preparing…'})
        group = group_from_job(symops, job['wyckoffTable'], str(job.get('spaceGroup', '')))
        formula = parse_formula(str(job['targetComposition']))
        rows, warnings = observation_rows(job)
        for w in warnings:
            self._log(w)
        plan, auto = z_plan(job, formula, group)
        if len(plan) > 1:
            self.post({'type': 'wy-info', 'message': f'Trying Z = {", ".join(str(z) for z in plan)}.'})
        seed = job.get('seed')
        seed = int(seed) if isinstance(seed, (int, float)) and not isinstance(seed, bool) else 20261026
        particles = int(job.get('swarmParticles') or DEFAULT_PARTICLES)
        generations = int(job.get('swarmIterations') or DEFAULT_GENERATIONS)
        restarts = int(job.get('swarmRestarts') or DEFAULT_RESTARTS)
        particles = max(8, (particles + 7) // 8 * 8)
        settings = {}
        if isinstance(job.get('polyProb'), (int, float)):
            settings['polyProb'] = float(job['polyProb'])
        solutions, failures = [], []
        for idx, Z in enumerate(plan):
            if self.stop_requested():
                break
            label = f'Z = {Z}' if len(plan) > 1 else ''
            self.post({'type': 'wy-start', 'message': f'Preparing {label}…' if label else 'Preparing…',
                       'z': Z, 'zIndex': idx + 1, 'zCount': len(plan)})
            try:
                problem, labels = problem_for_z(job, group, formula, Z, rows)
            except CombinatorialError as e:
                failures.append({'Z': Z, 'why': str(e)})
                if len(plan) == 1:
                    raise
                self._log(f'Z = {Z}: {e}')
                continue
            if len(plan) > 1:
                self.post({'type': 'wy-info', 'message': f'Searching Z = {Z}…'})
            sol = self._search_one(problem, labels, Z, idx, len(plan), particles, generations, restarts, seed,
                                   settings)
            if sol is not None:
                solutions.append(sol)
                self.post({'type': 'wy-partial', 'solution': sol})
        stopped = self.stop_requested()
        if not solutions:
            if failures and len(failures) == len(plan):
                raise JobError('; '.join(f'Z = {f["Z"]}: {f["why"]}' for f in failures))
            raise JobError('Stopped before any assignment produced a finite score, so there is nothing to show.'
                           if stopped else 'The Wyckoff search produced no sites.')
        solutions.sort(key=lambda s: (0, s['refinement']['R']) if s.get('refinement') else (1, -s['searchCC']))
        best = solutions[0]
        self.post({'type': 'wy-structure', 'results': {
            'sites': best['sites'], 'wyckoffResult': best, 'refinement': best.get('refinement'),
            'cell': job['cell'], 'nOps': len(symops),
            'symops': [o.get('xyz') if isinstance(o, dict) else o for o in symops if
                       (o.get('xyz') if isinstance(o, dict) else o)],
            'rawPeakCount': len(best['sites']), 'map': None, 'gridSize': None, 'originShift': None, 'hand': None,
            'symmetryCorrelation': None, 'originScore': None, 'source': 'wyckoff', 'z': best['z'],
            'solutions': solutions, 'zPlan': plan, 'zFailures': failures or None, 'zScan': None,
            'autoZ': auto, 'densityMin': job.get('densityMin'), 'densityMax': job.get('densityMax'),
            'seed': seed, 'stopped': stopped}})

    def _search_one(self, problem, labels, Z, idx, n_z, particles, generations, restarts, seed, settings):
        search = self.search
        if search is None:
            from .swarm_wyckoff import run_wyckoff_waves
            search = run_wyckoff_waves

        def progress(p: dict):
            msg = {'type': 'wy-progress', 'wave': p.get('wave', 1), 'waves': p.get('waves', 1),
                   'generation': p.get('generation'), 'generations': p.get('generations'),
                   'restart': p.get('restart', 1), 'restarts': p.get('restarts', 1),
                   'best': p.get('best'), 'cc': p.get('cc'), 'assignment': None, 'bestSites': None,
                   'stage': p.get('stage', 'search'), 'fraction': p.get('fraction'),
                   'z': Z, 'zIndex': idx + 1, 'zCount': n_z}
            A = p.get('assignment')
            if A is not None and p.get('coords') is not None:
                msg['assignment'] = [f'{el} {pos}' for el, pos in labels[A]]
                msg['bestSites'] = site_records(problem, A, p['coords'])
            self.post(msg)

        res = search(problem, particles, generations, restarts, seed, settings=settings or None,
                     on_progress=progress, should_stop=self.stop_requested, refine=True,
                     chunk=max(1, generations // PROGRESS_CHUNKS))
        if res.best_coords is None:
            return None
        A = int(res.best_assignment)
        coords = np.asarray(res.best_coords, dtype=np.float64)
        refinement = None
        ref = res.refined.get(A) if res.refined else None
        if ref and 'coords' in ref:
            coords = np.asarray(ref['coords'], dtype=np.float64)
            refinement = {'R': float(ref['r']), 'RStart': float(ref['r_start']), 'converged': bool(ref['converged'])}
        return {'z': Z, 'assignment': [f'{el} {pos}' for el, pos in labels[A]], 'assignmentIndex': A,
                'searchCC': float(res.best_cc), 'penalty': float(res.best_pen), 'refinement': refinement,
                'sites': site_records(problem, A, coords), 'ranked': True, 'unrefined': refinement is None,
                'stopped': self.stop_requested(), 'trials': int(res.trials),
                'perAssignment': {' + '.join(f'{el} {pos}' for el, pos in labels[a]): float(cc)
                                  for a, cc in res.per_assignment.items()},
                'cpuCheck': dict(res.cpu_check) if res.cpu_check else None}
