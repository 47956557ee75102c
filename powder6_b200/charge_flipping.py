"""Dual-space charge flipping on a powder reflection model, on the B200.

The host half of js/charge_flipping_worker.js (the reflection model, the
random starts, the weak-orbit classification, the run) over the C ABI of
``libp6cuda`` (``p6_cf_*``, csrc/cf.cu), which runs the cycle of
charge_flipping.wgsl:182-632 for any number of independent trials in the same
launches.

Names follow the reference: ``build_reflection_model`` (js/charge_flipping_
worker.js:563-948), ``model_initial_grid`` (:951-981),
``classify_weak_orbits`` (the rule of :1213-1310), ``find_systematic_absences``
(:336-424), ``normalize_symops`` (:279-298), ``run_charge_flipping``
(:1997-2500, the GPU run), and ``cf_plan`` (js/cf_adaptive.js:43-51, the
settings of the adaptive multi-start search, whose trials run here as one
batch).  Differences from the reference, each on purpose:

- The space group comes as its operators (``symops``); the reference's Laue
  class fallback without operators is not carried (a ``ValueError`` says so).
- The Lorentz-polarisation correction takes a per-peak ``lp`` when the peak
  has one (as the reference prefers), else the Bragg-Brentano form with the
  polarisation ratio K (``job['polarizationK']``, default 1: unpolarised).
- A reflection whose amplitude has collapsed restarts on a Philox draw keyed
  by (member, seed) instead of the reference's integer hash.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Dict, List, Optional, Sequence

import numpy as np

from ._lib import check, load
from .workloads import mulberry32   # the reference's seeded stream of random starts

IDX_MASK = 0x7FFFFFFF
CONJ_BIT = 0x80000000

# Lattice-centring translations (International Tables; R in the obverse
# hexagonal setting).
CENTRING_VECTORS = {
    'P': [],
    'A': [(0.0, 0.5, 0.5)],
    'B': [(0.5, 0.0, 0.5)],
    'C': [(0.5, 0.5, 0.0)],
    'I': [(0.5, 0.5, 0.5)],
    'F': [(0.0, 0.5, 0.5), (0.5, 0.0, 0.5), (0.5, 0.5, 0.0)],
    'R': [(2 / 3, 1 / 3, 1 / 3), (1 / 3, 2 / 3, 2 / 3)],
}


# ---------------------------------------------------------------------------
# Symmetry
# ---------------------------------------------------------------------------
def normalize_symops(raw) -> Optional[List[dict]]:
    """Operators {r (9, row-major), t (3)} with translations folded into
    [0, 1) and exact duplicates removed (js/charge_flipping_worker.js:279-298)."""
    if not raw:
        return None
    out, seen = [], set()
    for op in raw:
        if not op or len(op.get('r', ())) != 9:
            continue
        r = [float(v) for v in op['r']]
        t = [float(v) for v in op.get('t', (0, 0, 0))]
        if op.get('t_num') is not None and op.get('t_den'):
            t = [float(v) / float(op['t_den']) for v in op['t_num']]
        if not all(math.isfinite(v) for v in r + t):
            continue
        tw = []
        for v in t:
            f = v - math.floor(v)
            tw.append(0.0 if abs(f - 1) < 1e-9 else f)
        key = (tuple(r), tuple(round(v * 5040) for v in tw))
        if key in seen:
            continue
        seen.add(key)
        out.append({'r': [int(round(v)) for v in r], 't': tw})
    return out or None


def _row_apply(h, r):
    """(hR)_j = sum_i h_i R_ij, r row-major."""
    return (h[0] * r[0] + h[1] * r[3] + h[2] * r[6],
            h[0] * r[1] + h[1] * r[4] + h[2] * r[7],
            h[0] * r[2] + h[1] * r[5] + h[2] * r[8])


def find_systematic_absences(N: int, symops: Optional[List[dict]], centring: str = 'P') -> np.ndarray:
    """Grid indices of the extinct reflections: h is extinct when some
    operator (R, t) has hR = h and h.t not an integer; centring vectors are
    added to every rotation's translations whether or not the operator list
    carries them (js/charge_flipping_worker.js:336-424).  Vectorised over the
    whole signed index range of the grid."""
    cvecs = CENTRING_VECTORS.get(str(centring or 'P').upper(), [])
    if symops:
        by_rot: Dict[tuple, list] = {}
        for op in symops:
            by_rot.setdefault(tuple(op['r']), []).append(tuple(op['t']))
        if cvecs:
            def key(t):
                return tuple(round((v - math.floor(v)) * 5040) % 5040 for v in t)
            for r, ts in by_rot.items():
                seen = {key(t) for t in ts}
                for c in cvecs:
                    for t0 in list(ts):
                        t = (t0[0] + c[0], t0[1] + c[1], t0[2] + c[2])
                        if key(t) not in seen:
                            seen.add(key(t))
                            ts.append(t)
        rots = list(by_rot.items())
    else:
        if not cvecs:
            return np.zeros(0, np.uint32)
        rots = [((1, 0, 0, 0, 1, 0, 0, 0, 1), list(cvecs))]
    half = N >> 1
    m = np.arange(N)
    s = np.where(m > half, m - N, m)
    l, k, h = np.meshgrid(s, s, s, indexing='ij')       # flat index h + k N + l N^2
    h, k, l = h.ravel(), k.ravel(), l.ravel()
    extinct = np.zeros(N ** 3, bool)
    for r, ts in rots:
        hr = h * r[0] + k * r[3] + l * r[6]
        kr = h * r[1] + k * r[4] + l * r[7]
        lr = h * r[2] + k * r[5] + l * r[8]
        fixed = (hr == h) & (kr == k) & (lr == l)
        for t in ts:
            ht = h * t[0] + k * t[1] + l * t[2]
            extinct |= fixed & (np.abs(ht - np.round(ht)) > 1e-6)
    extinct[0] = False
    return np.nonzero(extinct)[0].astype(np.uint32)


def lorentz_polarization(tth: float, K: float = 1.0) -> float:
    """Bragg-Brentano Lp with polarisation ratio K (1 where the geometry is
    degenerate, the reference's lenient policy)."""
    if not (tth is not None and math.isfinite(tth) and 0 < tth < 180):
        return 1.0
    th = math.radians(tth / 2)
    s, c = math.sin(th), math.cos(th)
    if s < 1e-6 or c < 1e-6:
        return 1.0
    k = K if (K is not None and math.isfinite(K) and K >= 0) else 1.0
    c2 = math.cos(math.radians(tth))
    return (1 / (s * s * c)) * ((1 + k * c2 * c2) / (1 + k))


def overlap(a: dict, b: dict, tol_tth: float = 0.05, fwhm_fraction: float = 0.0) -> bool:
    """Two reflections measured as one peak (js/cf_adaptive.js:13-19)."""
    ta, tb = a.get('tth'), b.get('tth')
    if ta is not None and tb is not None and math.isfinite(ta) and math.isfinite(tb):
        tol = tol_tth
        fa, fb = a.get('fwhm'), b.get('fwhm')
        if fwhm_fraction and fwhm_fraction > 0 and fa and fb and fa > 0 and fb > 0 and math.isfinite(fa + fb):
            tol = fwhm_fraction * (fa + fb) / 2
        return abs(tb - ta) <= (tol if math.isfinite(tol) else 0.05)
    da, db = a.get('d'), b.get('d')
    return bool(da and db and da > 0 and db > 0 and abs(da - db) <= 1e-4 * da)


# ---------------------------------------------------------------------------
# The reflection model
# ---------------------------------------------------------------------------
def build_reflection_model(job: dict, N: int) -> dict:
    """Orbits, 2-theta clusters and the absent list on an N^3 grid
    (js/charge_flipping_worker.js:563-948): one orbit per unique reflection
    (its direct images first, then the Friedel mates of what is left, each
    member with the phase exp(+2 pi i h0.t) of the operator that produced
    it), intensities with Lp divided out and shared over the members that fit
    the grid, overlapping reflections clustered, systematically absent ones
    given no orbit (their intensity stays with an allowed cluster), grid
    points claimed once."""
    N2 = N * N
    symops = normalize_symops(job.get('symops'))
    if not symops:
        raise ValueError('charge flipping needs the space-group operators (symops); '
                         'the Laue-class fallback is not carried')
    absent = find_systematic_absences(N, symops, job.get('centering') or job.get('centring') or 'P')
    absent_set = set(absent.tolist())
    apply_lp = job.get('applyLP', True) is not False
    pol_k = job.get('polarizationK', 1.0)
    tol = job.get('overlapTolTth', 0.05)
    tol = tol if (tol is not None and math.isfinite(tol)) else 0.05
    fwhm_fraction = job.get('overlapFwhmFraction') or 0.0

    def wrap(v):
        return v % N

    dropped_zero = dropped_range = dropped_duplicate = 0
    max_index = 0
    refs = []
    for peak in job.get('hklList') or []:
        if not peak:
            continue
        I = peak.get('intensity')
        I = float(I) if I is not None else float('nan')
        if not math.isfinite(I) or I < 0:
            dropped_zero += 1
            continue
        h0, k0, l0 = peak.get('h_orig'), peak.get('k_orig'), peak.get('l_orig')
        if h0 is None or k0 is None or l0 is None:
            continue
        h0, k0, l0 = int(h0), int(k0), int(l0)
        if h0 == 0 and k0 == 0 and l0 == 0:
            continue
        positions: Dict[tuple, dict] = {}
        op_phases = []
        for op in symops:
            h, k, l = _row_apply((h0, k0, l0), op['r'])
            ht = h0 * op['t'][0] + k0 * op['t'][1] + l0 * op['t'][2]
            cr, ci = math.cos(2 * math.pi * ht), math.sin(2 * math.pi * ht)
            op_phases.append((h, k, l, cr, ci))
            positions.setdefault((h, k, l), {'h': h, 'k': k, 'l': l, 'cr': cr, 'ci': ci, 'conj': 0})
        for h, k, l, cr, ci in op_phases:
            positions.setdefault((-h, -k, -l), {'h': -h, 'k': -k, 'l': -l, 'cr': cr, 'ci': ci, 'conj': 1})
        m_true = len(positions)
        members, out_of_range = [], False
        for p in positions.values():
            m = max(abs(p['h']), abs(p['k']), abs(p['l']))
            max_index = max(max_index, m)
            if 2 * m >= N:
                out_of_range = True
                continue
            members.append(p)
        if out_of_range:
            dropped_range += 1
        if not members:
            continue
        sys_absent = any(wrap(p['h']) + wrap(p['k']) * N + wrap(p['l']) * N2 in absent_set for p in members)
        lp = 1.0
        if apply_lp:
            plp = peak.get('lp')
            lp = plp if (plp is not None and math.isfinite(plp) and plp > 0) else lorentz_polarization(
                peak.get('tth'), pol_k)
        mate = positions.get((-h0, -k0, -l0))
        centric = -0.5 * math.atan2(mate['ci'], mate['cr']) if (mate and not mate['conj']) else float('nan')
        raw = peak.get('rawIntensity')
        sigma = peak.get('sigma')
        fw = peak.get('fwhm')
        refs.append({'h0': h0, 'k0': k0, 'l0': l0, 'tth': peak.get('tth'), 'd': peak.get('d'),
                     'fwhm': fw if (fw is not None and fw > 0) else None, 'members': members, 'mTrue': m_true,
                     'centric': centric, 'targetI': (I / lp) * (len(members) / m_true), 'absent': sys_absent,
                     'rawI': float(raw) if raw is not None and math.isfinite(raw) else I,
                     'sigma': float(sigma) if sigma is not None and sigma > 0 else None})
    if not refs:
        return {'error': 'no-reflections', 'max_index_seen': max_index, 'min_grid_for_all': 2 * max_index + 2,
                'dropped_zero': dropped_zero, 'dropped_range': dropped_range}

    def sort_key(r):
        if r['tth'] is not None:
            return r['tth']
        return 1 / r['d'] if r['d'] else 0.0
    refs.sort(key=sort_key)
    cluster_of = [0] * len(refs)
    n_clusters = 0
    for i in range(1, len(refs)):
        if not overlap(refs[i - 1], refs[i], tol, fwhm_fraction):
            n_clusters += 1
        cluster_of[i] = n_clusters
    n_clusters += 1
    has_allowed = [False] * n_clusters
    for i, r in enumerate(refs):
        if not r['absent']:
            has_allowed[cluster_of[i]] = True
    significant_absent = 0
    for i, r in enumerate(refs):
        if r['absent'] and not has_allowed[cluster_of[i]] and r['sigma'] and r['rawI'] / r['sigma'] >= 3:
            significant_absent += 1
    requested_lambda = min(1.0, max(0.0, float(job.get('symLambda') or 0.0)))
    if requested_lambda >= 0.999 and significant_absent > 0:
        return {'error': 'significant-systematic-absence', 'significant_absent': significant_absent}

    orbit_start, orbit_count, orbit_target, orbit_centric = [], [], [], []
    idx_flat, phase_flat = [], []
    c_start, c_n, c_obs = [], [], []
    claimed = set()
    cur = -1
    for i, r in enumerate(refs):
        if cluster_of[i] != cur:
            cur = cluster_of[i]
            c_start.append(len(orbit_start))
            c_n.append(0)
            c_obs.append(0.0)
        c = len(c_start) - 1
        if r['absent']:
            c_obs[c] += r['targetI']
            continue
        start, count = len(idx_flat), 0
        for p in r['members']:
            gi = wrap(p['h']) + wrap(p['k']) * N + wrap(p['l']) * N2
            if gi in claimed:
                dropped_duplicate += 1
                continue
            claimed.add(gi)
            idx_flat.append((gi | CONJ_BIT) if p['conj'] else gi)
            phase_flat += [p['cr'], p['ci']]
            count += 1
        if count == 0:
            continue
        scaled = r['targetI'] * (count / len(r['members']))
        orbit_start.append(start)
        orbit_count.append(count)
        orbit_target.append(scaled)
        orbit_centric.append(r['centric'])
        c_n[c] += 1
        c_obs[c] += scaled
    if not orbit_start:
        return {'error': 'no-reflections', 'max_index_seen': max_index, 'min_grid_for_all': 2 * max_index + 2,
                'dropped_zero': dropped_zero, 'dropped_range': dropped_range}
    keep = [c for c in range(len(c_start)) if c_n[c] > 0]
    n_members = len(idx_flat)
    return {
        'N': N,
        'n_orbits': len(orbit_start), 'n_clusters': len(keep), 'n_members': n_members,
        'orbit_start': np.array(orbit_start, np.uint32), 'orbit_count': np.array(orbit_count, np.uint32),
        'orbit_target_i': np.array(orbit_target, np.float32), 'orbit_centric_phase': np.array(orbit_centric, np.float64),
        'orbit_idx': np.concatenate([np.array(idx_flat, np.uint32), absent]).astype(np.uint32),
        'phase': np.array(phase_flat, np.float32),
        'cluster_orbit_start': np.array([c_start[c] for c in keep], np.uint32),
        'cluster_n_orbits': np.array([c_n[c] for c in keep], np.uint32),
        'cluster_obs_i': np.array([c_obs[c] for c in keep], np.float32),
        'absent_start': n_members, 'absent_count': int(len(absent)),
        'dropped_zero': dropped_zero, 'dropped_range': dropped_range, 'dropped_duplicate': dropped_duplicate,
        'significant_absent': significant_absent, 'max_index_seen': max_index, 'min_grid_for_all': 2 * max_index + 2,
    }


def model_initial_grid(model: dict, N: int, seed: int) -> np.ndarray:
    """A random start that already obeys the space group
    (js/charge_flipping_worker.js:951-981): one phase per orbit (0 or pi
    from the centric phase for centric orbits), propagated by the members'
    phase factors, amplitude sqrt(target / count).  2 N^3 floats."""
    init = np.zeros(2 * N ** 3, np.float32)
    rand = mulberry32(seed)
    idx, ph = model['orbit_idx'], model['phase']
    for g in range(model['n_orbits']):
        start, count = int(model['orbit_start'][g]), int(model['orbit_count'][g])
        amp = math.sqrt(max(0.0, float(model['orbit_target_i'][g])) / count)
        u = rand()
        centric = float(model['orbit_centric_phase'][g])
        ang = centric + (0.0 if u < 0.5 else math.pi) if math.isfinite(centric) else 2 * math.pi * u
        f0r, f0i = amp * math.cos(ang), amp * math.sin(ang)
        for p in range(start, start + count):
            word = int(idx[p])
            i = word & IDX_MASK
            cr, ci = float(ph[2 * p]), float(ph[2 * p + 1])
            a = f0r * cr - f0i * ci
            b = f0r * ci + f0i * cr
            if word & CONJ_BIT:
                b = -b
            init[2 * i] = a
            init[2 * i + 1] = b
    return init


def classify_weak_orbits(model: dict, fraction: float, grouping: str = 'cluster') -> dict:
    """Orbits that take the quarter-turn instead of the amplitude constraint
    (the weak-reflection rule of js/charge_flipping_worker.js:1213-1310).

    The units ranked are single orbits (``grouping='individual'``) or whole
    2-theta clusters; a unit's strength is its observed intensity per grid
    point it occupies (a unit with no points ranks strongest).  The weakest
    floor(fraction * units) are flagged, every orbit of a flagged cluster
    with it.  Returns the per-orbit flags and a summary: the mode, the
    strength of the last unit flagged, and the flagged and total counts."""
    mode = 'individual' if grouping == 'individual' else 'cluster'
    frac = min(1.0, max(0.0, float(fraction or 0.0)))
    count = np.asarray(model['orbit_count'], dtype=np.float64)
    n_orb = int(model['n_orbits'])
    if mode == 'individual':
        intensity = np.asarray(model['orbit_target_i'], dtype=np.float64)
        points = count
    else:
        start = np.asarray(model['cluster_orbit_start'], dtype=np.int64)
        span = np.asarray(model['cluster_n_orbits'], dtype=np.int64)
        intensity = np.asarray(model['cluster_obs_i'], dtype=np.float64)
        # points per cluster: prefix sums of the orbit point counts over each span
        cum = np.concatenate([[0.0], np.cumsum(count)])
        points = cum[start + span] - cum[start]
    with np.errstate(divide='ignore', invalid='ignore'):
        strength = np.where(points > 0, intensity / np.where(points > 0, points, 1.0), np.inf)
    n_units = len(strength)
    n_weak = min(n_units, int(math.floor(frac * n_units)))
    weakest = np.argsort(strength, kind='stable')[:n_weak]
    if mode == 'individual':
        flags = np.zeros(n_orb, dtype=np.uint8)
        flags[weakest] = 1
    else:
        # mark each flagged cluster's orbit span with a difference array
        edge = np.zeros(n_orb + 1, dtype=np.int64)
        np.add.at(edge, start[weakest], 1)
        np.add.at(edge, start[weakest] + span[weakest], -1)
        flags = (np.cumsum(edge)[:n_orb] > 0).astype(np.uint8)
    return {'flags': flags, 'mode': mode, 'cutoff': float(strength[weakest[-1]]) if n_weak else 0.0,
            'weak_units': n_weak, 'total_units': n_units, 'weak_orbits': int(flags.sum())}


MIN_STARTS, MAX_STARTS = 6, 128


def cf_plan(starts: int, difficult: bool = False, have_symmetry: bool = True) -> dict:
    """Settings of the adaptive multi-start search (js/cf_adaptive.js:43-51):
    three (threshold, weak fraction, symmetry weight) settings, assigned to
    the starts in turn; every start is one trial of the same batch here."""
    if not (MIN_STARTS <= int(starts) <= MAX_STARTS):
        raise ValueError(f'adaptive charge flipping needs {MIN_STARTS}-{MAX_STARTS} random starts')
    settings = ([{'threshold': 1.0, 'weakFraction': .25, 'symLambda': .5},
                 {'threshold': 1.1, 'weakFraction': .15, 'symLambda': .5},
                 {'threshold': 1.2, 'weakFraction': .25, 'symLambda': .75}] if difficult else
                [{'threshold': 1.0, 'weakFraction': .1, 'symLambda': 0.0},
                 {'threshold': 1.1, 'weakFraction': .15, 'symLambda': .5},
                 {'threshold': 1.2, 'weakFraction': .2, 'symLambda': .5}])
    for i, s in enumerate(settings):
        s['id'] = i + 1
        if not have_symmetry:
            s['symLambda'] = 0.0
        s['starts'] = 0
    trials = []
    for i in range(int(starts)):
        s = settings[i % len(settings)]
        s['starts'] += 1
        trials.append(dict(s, seedSlot=i // len(settings)))
    return {'version': 1, 'settings': settings, 'trials': trials, 'difficult': bool(difficult)}


# ---------------------------------------------------------------------------
# The device session
# ---------------------------------------------------------------------------
class P6CfModel(C.Structure):
    _fields_ = [('n', C.c_int), ('n_orbits', C.c_int), ('orbit_start', C.c_void_p), ('orbit_count', C.c_void_p),
                ('n_members', C.c_int), ('orbit_idx', C.c_void_p), ('phase', C.c_void_p),
                ('n_clusters', C.c_int), ('cluster_orbit_start', C.c_void_p), ('cluster_n_orbits', C.c_void_p),
                ('cluster_obs_i', C.c_void_p), ('n_absent', C.c_int), ('absent_idx', C.c_void_p)]


class P6CfTrial(C.Structure):
    _fields_ = [('delta_sigma', C.c_float), ('sym_lambda', C.c_float), ('seed', C.c_uint32), ('weak', C.c_void_p)]


class CFSession:
    """All trials of one reflection model on one device.  ``trials`` is a
    list of {'threshold' (delta in sigma), 'symLambda', 'seed', 'weak'
    (n_orbits flags or None)}."""

    def __init__(self, model: dict, trials: Sequence[dict], device: int = 0):
        self.lib = load()
        self.N = int(model['N'])
        self.n_trials = len(trials)
        self.model = model
        self._keep = []

        def a(x, dt):
            x = np.ascontiguousarray(x, dtype=dt)
            self._keep.append(x)
            return x.ctypes.data

        nm = model['n_members']
        m = P6CfModel()
        m.n = self.N
        m.n_orbits = model['n_orbits']
        m.orbit_start = a(model['orbit_start'], np.uint32)
        m.orbit_count = a(model['orbit_count'], np.uint32)
        m.n_members = nm
        m.orbit_idx = a(model['orbit_idx'][:nm], np.uint32)
        m.phase = a(model['phase'], np.float32)
        m.n_clusters = model['n_clusters']
        m.cluster_orbit_start = a(model['cluster_orbit_start'], np.uint32)
        m.cluster_n_orbits = a(model['cluster_n_orbits'], np.uint32)
        m.cluster_obs_i = a(model['cluster_obs_i'], np.float32)
        m.n_absent = model['absent_count']
        m.absent_idx = a(model['orbit_idx'][nm:], np.uint32) if model['absent_count'] else None
        arr = (P6CfTrial * self.n_trials)()
        for t, tr in enumerate(trials):
            arr[t].delta_sigma = float(tr.get('threshold', 1.1))
            arr[t].sym_lambda = float(tr.get('symLambda', 0.0))
            arr[t].seed = int(tr.get('seed', 0)) & 0xFFFFFFFF
            w = tr.get('weak')
            arr[t].weak = a(w, np.uint8) if w is not None else None
        h = C.c_void_p()
        check(self.lib.p6_cf_create(C.byref(m), self.n_trials, arr, int(device), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, 'h', None):
            self.lib.p6_cf_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_grid(self, grid: np.ndarray, trial: int = -1):
        g = np.ascontiguousarray(grid, dtype=np.float32)
        assert g.size == 2 * self.N ** 3
        check(self.lib.p6_cf_set_grid(self.h, int(trial), g.ctypes.data))

    def run(self, cycles: int) -> np.ndarray:
        """R of every cycle of every trial (n_trials x cycles)."""
        hist = np.zeros((self.n_trials, max(1, cycles)), np.float32)
        check(self.lib.p6_cf_run(self.h, int(cycles), hist.ctypes.data))
        return hist[:, :cycles]

    def best_r(self) -> np.ndarray:
        out = np.zeros(self.n_trials, np.float32)
        check(self.lib.p6_cf_best_r(self.h, out.ctypes.data))
        return out

    def read(self, trial: int, which: str = 'current') -> np.ndarray:
        """'current' / 'best': the F grid (2 N^3 floats); 'map': the density of
        the best grid (N^3 floats)."""
        code = {'current': 0, 'best': 1, 'map': 2}[which]
        out = np.zeros((self.N ** 3) * (1 if code == 2 else 2), np.float32)
        check(self.lib.p6_cf_read(self.h, int(trial), code, out.ctypes.data))
        return out

    def last_ms(self) -> float:
        ms = C.c_float()
        check(self.lib.p6_cf_last_ms(self.h, C.byref(ms)))
        return ms.value

    def time_kernels(self, cycles: int = 3):
        """Mean device ms of one transform pass and of one reciprocal step
        (the cycles run for real; their R factors are not recorded)."""
        a, b = C.c_float(), C.c_float()
        check(self.lib.p6_cf_time_kernels(self.h, int(cycles), C.byref(a), C.byref(b)))
        return a.value, b.value

    def launch_count(self) -> int:
        n = C.c_longlong()
        check(self.lib.p6_cf_launch_count(self.h, C.byref(n)))
        return n.value


def run_charge_flipping(job: dict, device: int = 0, trials: Optional[Sequence[dict]] = None) -> dict:
    """The GPU run of js/charge_flipping_worker.js:1997-2500 for one job
    (gridSize, maxIterations, thresholdSigma, seed, symops, symLambda,
    weakFraction, weakGrouping, hklList, ...), or for a batch of ``trials``
    ({'threshold', 'symLambda', 'weakFraction', 'seed'}; the job supplies what
    a trial leaves out), all in the same launches.  Returns the reference's
    result fields for the best trial, and ``trials`` with every trial's."""
    N = int(job['gridSize'])
    model = build_reflection_model(job, N)
    if 'error' in model:
        raise ValueError(f"reflection model: {model['error']}")
    cycles = int(job.get('maxIterations', 100))
    base = {'threshold': float(job.get('thresholdSigma', 1.1)),
            'symLambda': min(1.0, max(0.0, float(job.get('symLambda') or 0.0))),
            'weakFraction': float(job.get('weakFraction') or 0.0), 'seed': int(job.get('seed', 1))}
    specs = []
    for t in (trials or [{}]):
        spec = dict(base, **t)
        if 'seed' not in t and 'seedSlot' in t:
            # the seed of an adaptive start (js/rietveld/rv_solve.js:556)
            spec['seed'] = (base['seed'] + int(t['seedSlot']) * 7919) & 0xFFFFFFFF
        specs.append(spec)
    grouping = job.get('weakGrouping', 'cluster')
    dev_trials, weak_counts = [], []
    for t in specs:
        wk = classify_weak_orbits(model, t['weakFraction'], grouping)
        weak_counts.append(wk['weak_orbits'])
        dev_trials.append({'threshold': t['threshold'], 'symLambda': t['symLambda'], 'seed': t['seed'],
                           'weak': wk['flags'] if wk['weak_orbits'] else None})
    with CFSession(model, dev_trials, device) as s:
        for i, t in enumerate(specs):
            s.set_grid(model_initial_grid(model, N, t['seed']), i)
        hist = s.run(cycles)
        best = s.best_r()
        results = []
        for i, t in enumerate(specs):
            h = hist[i]
            fin = np.isfinite(h)
            best_iter = int(np.argmin(np.where(fin, h, np.inf))) + 1 if fin.any() else 0
            results.append({'bestR': float(best[i]), 'bestIter': best_iter, 'finalR': float(h[-1]) if cycles else math.nan,
                            'rHistory': h, 'seed': t['seed'], 'symLambda': t['symLambda'],
                            'threshold': t['threshold'], 'weak_orbits': weak_counts[i]})
        top = int(np.argmin(best))
        out = dict(results[top])
        out.update({'map': s.read(top, 'map'), 'backend': 'gpu', 'trials': results, 'bestTrial': top,
                    'gridSize': N, 'n_orbits': model['n_orbits'], 'n_clusters': model['n_clusters'],
                    'deviceMs': s.last_ms()})
    return out


# ---------------------------------------------------------------------------
# A synthetic job (test and benchmark input)
# ---------------------------------------------------------------------------
def synthetic_job(group_number: int = 14, cell: Optional[dict] = None, atoms: Optional[Sequence[tuple]] = None,
                  grid: int = 32, dmin: float = 1.0, wavelength: float = 1.5406, overlap_tol: float = 0.02,
                  biso: float = 1.5, seed: int = 1, **job) -> dict:
    """A charge-flipping job from a known structure: the unique reflections
    of ``group_number`` in ``cell`` down to ``dmin`` (those that fit the
    grid), intensity m |F|^2 with point scatterers of weight Z and an
    isotropic displacement exp(-B s^2), 2-theta at ``wavelength``, no Lp.
    ``atoms`` are (x, y, z, Z) in the asymmetric unit; the default is four
    light and one heavy site drawn from ``seed``."""
    from .reflections import generate_reflections
    from .symmetry import space_group
    g = space_group(group_number)
    cell = cell or {'a': 9.1, 'b': 7.3, 'c': 10.4, 'alpha': 90.0, 'beta': 104.0, 'gamma': 90.0}
    if atoms is None:
        rng = np.random.default_rng(seed)
        atoms = [tuple(rng.uniform(0, 1, 3)) + (z,) for z in (26.0, 8.0, 8.0, 7.0, 6.0)]
    refl = generate_reflections(cell, g.ops, dmin)
    hkl = np.array([[r.h, r.k, r.l] for r in refl], dtype=np.float64)
    d = np.array([r.d0 for r in refl])
    s2 = 1.0 / (4 * d * d)
    F = np.zeros(len(refl), np.complex128)
    for x, y, z, Z in atoms:
        for o in g.ops:
            p = np.array([sum(o.r[3 * i + k] * (x, y, z)[k] for k in range(3)) + o.t_frac[i] for i in range(3)])
            F += Z * np.exp(-biso * s2) * np.exp(2j * np.pi * (hkl @ (p - np.floor(p))))
    peaks = []
    for r, f, dd in zip(refl, F, d):
        if 2 * max(abs(r.h), abs(r.k), abs(r.l)) >= grid:
            continue
        st = wavelength / (2 * dd)
        if st >= 1:
            continue
        peaks.append({'h_orig': r.h, 'k_orig': r.k, 'l_orig': r.l, 'intensity': float(r.m * abs(f) ** 2),
                      'tth': 2 * math.degrees(math.asin(st)), 'd': float(dd), 'multiplicity': r.m})
    out = {'gridSize': grid, 'maxIterations': 100, 'thresholdSigma': 1.1, 'seed': seed, 'cell': cell,
           'symops': g.op_dicts(), 'symLambda': 0.5, 'weakFraction': 0.15, 'weakGrouping': 'cluster',
           'overlapTolTth': overlap_tol, 'applyLP': False, 'hklList': peaks, 'atoms': list(atoms),
           'groupNumber': group_number}
    out.update(job)
    return out
