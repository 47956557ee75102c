"""Reflection enumeration, observation grouping and the scattering table.

* ``generate_reflections`` follows ``generateReflections`` (js/rietveld_core.js:
  247-276) with ``laueRotations`` (:182-188) and ``isAllowed`` (:192-201): one
  reflection per Laue orbit (Friedel pairs merged), the canonical member being
  the one with the most non-negative indices and then the largest (h, k, l),
  systematic absences decided exactly from the operators, multiplicity = orbit
  size, sorted by d descending then h, k, l descending.  Vectorised with numpy;
  the float operations that decide the cutoff and the sort are the reference's,
  in its order.
* ``pack_reflections`` follows ``swPackReflections`` (js/swarm_wyckoff.js:
  423-620) with ``obsGroupVariance`` (js/observations.js:350-371): lines closer
  than the overlap tolerance become one observation, hkl packed 10 bits each
  (biased by 512), ``groupMeta`` = [start, count, sum(mult Fo^2), weight], weights
  normalised to mean 1 and groups without a usable sigma dropped (weight 0).
* ``scattering_table`` follows ``swScatteringTable`` (js/swarm_wyckoff.js:
  891-915): f(s) exp(-B s^2/4) per (reflection, element), float32.
* ``ramped_group_count`` follows ``rampedGroupCount`` (js/swarm_wyckoff.js:
  934-938).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from .crystal import build_inv_dsq
from .symmetry import SymOp, TDEN, laue_rotations


@dataclass
class Reflection:
    h: int
    k: int
    l: int
    m: int
    d0: float
    eq: np.ndarray  # orbit members, (m, 3) int16


def generate_reflections(cell: Dict[str, float], ops: Sequence[SymOp], dmin: float,
                         box: Optional[Sequence[int]] = None, with_eq: bool = True) -> List[Reflection]:
    f = build_inv_dsq(cell)
    if f is None or not dmin > 0:
        return []
    lim = 1.0 / (dmin * dmin) * (1 + 1e-9)
    rots = np.array(laue_rotations(ops), dtype=np.int64).reshape(-1, 3, 3)
    if box is not None:
        hmax, kmax, lmax = (int(v) for v in box)
    else:
        hmax = math.floor(float(cell['a']) / dmin)
        kmax = math.floor(float(cell.get('b') or cell['a']) / dmin)
        lmax = math.floor(float(cell.get('c') or cell['a']) / dmin)
    hh, kk, ll = np.meshgrid(np.arange(-hmax, hmax + 1), np.arange(-kmax, kmax + 1),
                             np.arange(-lmax, lmax + 1), indexing='ij')
    H = np.stack([hh.ravel(), kk.ravel(), ll.ravel()], axis=1).astype(np.int64)
    H = H[np.any(H != 0, axis=1)]
    hf = H.astype(np.float64)
    q = inv_dsq_arr(f, hf[:, 0], hf[:, 1], hf[:, 2])
    keep = q > 0
    if box is None:
        keep &= q <= lim
    H, q = H[keep], q[keep]
    # orbit under the Laue group, h' = h R (row vector times matrix)
    V = np.einsum('nj,rjk->nrk', H, rots)                      # (n, nrot, 3)
    npos = (V >= 0).sum(axis=2)
    # canonical: max over (npos, h, k, l) lexicographic
    B = 1 << 12
    key = ((npos.astype(np.int64) * B + (V[:, :, 0] + 2048)) * B + (V[:, :, 1] + 2048)) * B + (V[:, :, 2] + 2048)
    best = np.argmax(key, axis=1)
    canon = V[np.arange(len(H)), best]
    is_canon = np.all(canon == H, axis=1)
    H, q, V = H[is_canon], q[is_canon], V[is_canon]
    # systematic absences: an operator with hR = h and h.t not an integer
    allowed = np.ones(len(H), dtype=bool)
    for o in ops:
        R = np.array(o.r, dtype=np.int64).reshape(3, 3)
        hr = H @ R
        fixed = np.all(hr == H, axis=1)
        p = H @ np.array(o.t, dtype=np.int64)          # in units of 1/TDEN
        allowed &= ~(fixed & (p % TDEN != 0))
    H, q, V = H[allowed], q[allowed], V[allowed]
    # multiplicity = number of distinct orbit members
    okey = ((V[:, :, 0] + 2048) * B + (V[:, :, 1] + 2048)) * B + (V[:, :, 2] + 2048)
    okey.sort(axis=1)
    mult = 1 + (np.diff(okey, axis=1) != 0).sum(axis=1)
    d0 = 1.0 / np.sqrt(q)
    order = np.lexsort((-H[:, 2], -H[:, 1], -H[:, 0], -d0))
    out = []
    for i in order:
        eq = None
        if with_eq:
            uniq = []
            seen = set()
            for r in range(V.shape[1]):
                t = (int(V[i, r, 0]), int(V[i, r, 1]), int(V[i, r, 2]))
                if t not in seen:
                    seen.add(t)
                    uniq.append(t)
            eq = np.array(uniq, dtype=np.int16)
        out.append(Reflection(int(H[i, 0]), int(H[i, 1]), int(H[i, 2]), int(mult[i]), float(d0[i]), eq))
    return out


def inv_dsq_arr(f, h, k, l):
    return ((((h * h * f['aa'] + k * k * f['bb']) + l * l * f['cc']) + h * k * f['ab']) + k * l * f['bc']) \
        + h * l * f['ac']


def centring_allowed(h: int, k: int, l: int, centring: Sequence[Sequence[float]]) -> bool:
    for c in centring:
        p = h * c[0] + k * c[1] + l * c[2]
        if abs(p - round(p)) >= 1e-6:
            return False
    return True


def obs_group_variance(members: Sequence[dict]) -> Optional[float]:
    v = 0.0
    by_hkl = {}
    for r in members:
        s = r.get('sigma')
        if not (s is not None and math.isfinite(s) and s > 0):
            return None
        sm = r['mult'] * s
        v += sm * sm
        by_hkl[(r['h'], r['k'], r['l'])] = r
    if not v > 0:
        return None
    c = 0.0
    if len(members) > 1:
        for r in members:
            for p in r.get('cov') or []:
                o = by_hkl.get((p[0], p[1], p[2]))
                if o is not None and o is not r and math.isfinite(p[3]):
                    c += 2 * r['mult'] * o['mult'] * p[3]
    return max(v + c, 1e-3 * v)


@dataclass
class PackedReflections:
    refl_pack: np.ndarray     # uint32 (2 * nRefl): packed hkl, multiplicity
    group_meta: np.ndarray    # float32 (4 * nGroups): start, count, Iobs, weight
    group_d: np.ndarray       # float32 (nGroups): 1/d of the group's first line
    refl_s: np.ndarray        # float32 (nRefl): 1/d per packed reflection
    n_refl: int
    n_groups: int
    group_stride: int = 4
    weighted: bool = False
    grouped_by: str = 'd-tolerance'
    problems: List[str] = field(default_factory=list)


def pack_reflections(rows: Sequence[dict], overlap_tol: float = 0.002,
                     fwhm_at: Optional[Callable[[float], float]] = None,
                     overlap_fwhm_frac: float = 0.5) -> PackedReflections:
    tol = overlap_tol
    sorted_rows = sorted(rows, key=lambda r: -r['d'])       # stable, like Array.prototype.sort
    groups: List[dict] = []
    cur = None
    width_misses = 0
    for r in sorted_rows:
        rt = r.get('tth', r.get('twoTheta', float('nan')))
        rt = float(rt) if rt is not None else float('nan')
        if cur is not None and fwhm_at is not None and math.isfinite(rt) and math.isfinite(cur['lastTth']):
            w = fwhm_at(rt)
            if w is not None and math.isfinite(w) and w > 0:
                same = abs(rt - cur['lastTth']) < overlap_fwhm_frac * w
            else:
                same = abs(r['d'] - cur['d']) / cur['d'] < tol
                width_misses += 1
        else:
            same = cur is not None and abs(r['d'] - cur['d']) / cur['d'] < tol
        if same:
            cur['members'].append(r)
            if math.isfinite(rt):
                cur['lastTth'] = rt
        else:
            cur = {'members': [r], 'd': r['d'], 'tth': rt, 'lastTth': rt}
            groups.append(cur)
    n_groups = len(groups)
    n_refl = len(sorted_rows)
    refl_pack = np.zeros(2 * n_refl, dtype=np.uint32)
    meta = np.zeros(4 * n_groups, dtype=np.float32)
    group_d = np.zeros(n_groups, dtype=np.float32)
    refl_s = np.zeros(n_refl, dtype=np.float32)
    n_unweighted = 0
    w = 0
    for gi, g in enumerate(groups):
        io = 0.0
        meta[4 * gi] = w
        meta[4 * gi + 1] = len(g['members'])
        for r in g['members']:
            if abs(r['h']) > 511 or abs(r['k']) > 511 or abs(r['l']) > 511:
                raise ValueError(f"Reflection {r['h']} {r['k']} {r['l']} exceeds the +/-511 packing range.")
            refl_pack[2 * w] = ((r['h'] + 512) & 0x3FF) | (((r['k'] + 512) & 0x3FF) << 10) | \
                (((r['l'] + 512) & 0x3FF) << 20)
            refl_pack[2 * w + 1] = r['mult']
            refl_s[w] = 1.0 / r['d']
            io += r['mult'] * r['Fo2']
            w += 1
        var = obs_group_variance(g['members'])
        meta[4 * gi + 2] = io
        if var is not None and var > 0:
            meta[4 * gi + 3] = 1.0 / var
        else:
            meta[4 * gi + 3] = 0.0
            n_unweighted += 1
        group_d[gi] = 1.0 / g['d']
    wsum, wn = 0.0, 0
    for gi in range(n_groups):
        v = float(meta[4 * gi + 3])
        if v > 0:
            wsum += v
            wn += 1
    if wn > 0:
        mean = wsum / wn
        for gi in range(n_groups):
            v = float(meta[4 * gi + 3])
            meta[4 * gi + 3] = v / mean if v > 0 else 0.0
    else:
        meta[3::4] = 1.0
    problems = []
    if n_unweighted and wn > 0:
        problems.append(f'{n_unweighted} of {n_groups} group(s) carry no usable standard uncertainty and were DROPPED.')
    grouped = ('profile-width' if (fwhm_at and width_misses == 0) else
               ('profile-width-partial' if fwhm_at else 'd-tolerance'))
    return PackedReflections(refl_pack, meta, group_d, refl_s, w, n_groups, 4, wn > 0, grouped, problems)


def unpack_hkl(pk: int):
    return ((pk & 0x3FF) - 512, ((pk >> 10) & 0x3FF) - 512, ((pk >> 20) & 0x3FF) - 512)


def scattering_table(refl: PackedReflections, demand: Sequence[dict],
                     form_factor: Callable[[str, float], Optional[float]], overall_b: float = 0.0):
    """float32 (nRefl * nElem) table of f(s) exp(-B s^2/4), s = 1/d."""
    n_elem = len(demand)
    table = np.zeros(refl.n_refl * n_elem, dtype=np.float32)
    s_of = np.zeros(refl.n_refl, dtype=np.float32)
    gs = refl.group_stride
    for g in range(refl.n_groups):
        st, c = int(refl.group_meta[g * gs]), int(refl.group_meta[g * gs + 1])
        for m in range(c):
            s_of[st + m] = refl.refl_s[st + m] if refl.refl_s[st + m] > 0 else refl.group_d[g]
    missing = set()
    for r in range(refl.n_refl):
        s = float(s_of[r])
        dw = math.exp(-overall_b * s * s / 4) if overall_b > 0 else 1.0
        for e in range(n_elem):
            fv = form_factor(demand[e]['element'], s)
            if fv is None or not math.isfinite(fv):
                fv = demand[e]['z']
                missing.add(demand[e]['element'])
            table[r * n_elem + e] = fv * dw
    return table, n_elem, sorted(missing)


def gaussian_form_factor(table: Dict[str, dict]) -> Callable[[str, float], Optional[float]]:
    """(element, s) -> f0(s) from five-Gaussian coefficients, stol = s/2 (js/scatterers.js:91-107, 142-185)."""
    by_key = {k.upper(): v for k, v in table.items()}

    def ff(element: str, s: float):
        e = by_key.get(str(element).upper())
        if e is None:
            return None
        stol = s / 2
        q = stol * stol
        f = e.get('c', 0.0) or 0.0
        for a, b in zip(e['a'], e['b']):
            f += a * math.exp(-b * q)
        return f
    return ff


def ramped_group_count(n_groups: int, generation: int, max_gen: int, start_frac: float = 0.25,
                       full_by: float = 0.6) -> int:
    t = min(1.0, generation / max(1.0, max_gen * full_by))
    frac = start_frac + (1 - start_frac) * t
    return max(8, min(n_groups, int(math.floor(n_groups * frac + 0.5))))
