"""Wyckoff assignments consistent with a composition: the caller of the
search that decides which (element, Wyckoff position) sets the device
searches.

Restates js/wyckoff_assign.js:184-206 (``multisets_summing_to``), :226-352
(site stabiliser, inversion and coordination compatibility), :354-572
(``enumerate_assignments``), :574-605 (the fixed-point clash message) and
:664-754 (``normalizer_permutations``, ``dedupe_equivalent_assignments``),
over this package's space groups (``symmetry.SpaceGroup``).  An enumerated
assignment converts to the search's ``wyckoff_tables.Assignment`` with
``to_search_assignment``.

Positions are the group's ``wyckoff`` list; ``demand`` is
[{'element', 'count' (atoms per cell), 'z', 'r'}].  Messages name the
constraint that failed, as the reference's do.
"""
from __future__ import annotations

import math
from typing import Dict, List, Optional, Sequence

from .symmetry import SpaceGroup, WyckoffPosition

MAX_SITES = 32            # sites one assignment may hold (the search kernel's limit)
MAX_ASSIGNMENTS = 4000    # enumeration cap

# A deliberately generic point: its projection onto a position cannot land on
# a higher-symmetry sub-position by accident.
_GENERIC = (0.1357913, 0.2468135, 0.3579246)

# Coordination polyhedra without an inversion centre.
NON_CENTROSYMMETRIC_GEOMETRY = {'tetrahedral', 'trigonal-planar', 'trigonal-pyramidal', 'square-pyramidal',
                                'trigonal-prismatic', 'see-saw', 'bent'}

# Central atoms for which four neighbours mean a tetrahedron (oxoanion and
# framework formers; four-coordinate d8 cations and O are often square planar).
TETRAHEDRAL_AT_FOUR = {'B', 'C', 'N', 'F', 'AL', 'SI', 'P', 'S', 'CL', 'GA', 'GE', 'AS', 'SE', 'BR', 'V', 'CR', 'MN',
                       'FE', 'CO', 'ZN', 'MO', 'W', 'TC', 'RE', 'BE', 'I', 'XE'}


def _ops(group: SpaceGroup):
    return [(tuple(o.r), tuple(o.t_frac)) for o in group.ops]


def multisets_summing_to(positions: Sequence[WyckoffPosition], target: int, opts: dict) -> List[List[int]]:
    """Index multisets of ``positions`` whose multiplicities sum to
    ``target``: a position without free coordinates at most once, one with
    free coordinates at most ``maxRepeat`` times, at most ``maxSites`` sites,
    at most ``maxPerElement`` results, indices non-decreasing."""
    out: List[List[int]] = []
    counts = [0] * len(positions)
    chosen: List[int] = []

    def rec(start: int, remaining: int):
        if remaining == 0:
            out.append(list(chosen))
            return
        if len(chosen) >= opts['maxSites'] or len(out) >= opts['maxPerElement']:
            return
        for i in range(start, len(positions)):
            m = positions[i].multiplicity
            if not m or m > remaining:
                continue
            cap = opts['maxRepeat'] if positions[i].n_free > 0 else 1
            if counts[i] >= cap:
                continue
            counts[i] += 1
            chosen.append(i)
            rec(i, remaining - m)
            chosen.pop()
            counts[i] -= 1
            if len(out) >= opts['maxPerElement']:
                return

    rec(0, target)
    return out


def _near_int(d: float, tol: float) -> bool:
    return abs(d - round(d)) < tol


def site_stabilizer(w: WyckoffPosition, ops) -> list:
    """Operators mapping the position's generic representative onto itself
    modulo a lattice translation."""
    p = w.project(*_GENERIC)
    stab = []
    for r, t in ops:
        q = [r[3 * i] * p[0] + r[3 * i + 1] * p[1] + r[3 * i + 2] * p[2] + t[i] for i in range(3)]
        if all(_near_int(q[i] - p[i], 1e-4) for i in range(3)):
            stab.append((r, t))
    return stab


def site_has_inversion(w: WyckoffPosition, ops) -> bool:
    return any(tuple(r) == (-1, 0, 0, 0, -1, 0, 0, 0, -1) for r, _ in site_stabilizer(w, ops))


def coordination_compatible(w: WyckoffPosition, element: str, req: Optional[dict], ops) -> Optional[str]:
    """None when an atom of ``element`` with coordination ``req`` ({'count',
    'geometry'}) can sit on ``w``; else the reason.  Parity: an inversion
    centre pairs every neighbour, so the count must be even.  Geometry: a
    polyhedron without an inversion centre (stated, or tetrahedral for the
    tetrahedral formers at four neighbours) cannot sit on one."""
    if not req or not req.get('count') or req['count'] <= 0 or not ops:
        return None
    if not site_has_inversion(w, ops):
        return None
    label = f'{w.multiplicity}{w.letter}'
    if req['count'] % 2 == 1:
        return (f"{element} needs {req['count']} neighbours, an odd number, but {label} has an inversion "
                f"centre, which pairs every neighbour with an antipode.")
    geom = str(req['geometry']).lower() if req.get('geometry') else None
    if not geom and req['count'] == 4 and str(element).upper() in TETRAHEDRAL_AT_FOUR:
        geom = 'tetrahedral'
    if geom and geom in NON_CENTROSYMMETRIC_GEOMETRY:
        return (f"{element} on {label} would put a {geom} coordination on an inversion centre, which no {geom} "
                f"arrangement has.")
    return None


def _fixed_point_clash(wyckoff, demand, per_element, fixed_only) -> Optional[str]:
    forced, pool = [], set()
    for e, combos in enumerate(per_element):
        if combos and all(any(i in fixed_only for i in c) for c in combos):
            forced.append(e)
            for c in combos:
                pool.update(i for i in c if i in fixed_only)
    if len(forced) < 2:
        return None

    def lst(a):
        return ''.join(a) if len(a) <= 1 else ', '.join(a[:-1]) + ' and ' + a[-1]
    who = [f"{demand[e]['element']} ({demand[e]['count']} per cell)" for e in forced]
    where = [f'{wyckoff[i].multiplicity}{wyckoff[i].letter}' for i in sorted(pool)]
    tail = (f'That is {len(forced)} elements for {len(pool)} such position(s). ' if len(forced) > len(pool)
            else 'No way of sharing them out leaves every element its own. ')
    return (f"No assignment places {lst([demand[e]['element'] for e in forced])} on separate sites: {lst(who)} can "
            f"only go on fixed points (positions with no free coordinate: {lst(where)}), and a fixed point holds "
            f"one element. " + tail + "The search builds ordered models, one element per site.")


def enumerate_assignments(group: SpaceGroup, demand: Sequence[dict], options: Optional[dict] = None) -> dict:
    """Every assignment of Wyckoff positions to the demanded atoms per cell
    (js/wyckoff_assign.js:354-572): per element, the multisets of positions
    summing to its count (largest multiplicities first, site-symmetry
    exclusions from ``coordination`` applied before the combinatorics), then
    their combinations with no fixed point shared by two elements and at most
    ``maxTotalSites`` sites.  Returns {'assignments': [{'sites': [{'element',
    'elementIdx', 'z', 'r', 'wIdx'}], 'nSites'}], 'truncated',
    'droppedTooManySites', 'siteSymmetryExcluded'} or, when none exists, an
    empty list with an 'error' naming the cause."""
    options = dict(options or {})
    wyckoff = group.wyckoff
    ops = _ops(group)
    ceiling = options.get('ceiling', 24)
    mults = [w.multiplicity for w in wyckoff if w.multiplicity > 0]
    m_max = max(mults) if mults else 1
    max_count = max((d['count'] for d in demand), default=0)
    needed = min(ceiling, math.ceil(max_count / m_max))
    opts = {'maxSites': min(ceiling, max(options.get('maxSites', 4), needed)),
            'maxRepeat': min(ceiling, max(options.get('maxRepeat', 4), needed)),
            'maxPerElement': options.get('maxPerElement', 500),
            'maxTotal': options.get('maxTotal', MAX_ASSIGNMENTS)}
    max_total_sites = options.get('maxTotalSites', MAX_SITES)
    idx = sorted(range(len(wyckoff)), key=lambda i: -wyckoff[i].multiplicity)   # stable, as the reference's sort
    srt = [wyckoff[i] for i in idx]
    coordination = options.get('coordination')
    use_ops = ops if options.get('symOps', True) else None
    excluded: List[str] = []
    excluded_for: List[list] = [[] for _ in demand]
    allowed_for: List[Optional[set]] = []
    for e, d in enumerate(demand):
        req = coordination.get(str(d['element']).upper()) if coordination else None
        if not req or not use_ops:
            allowed_for.append(None)
            continue
        ok = set()
        for i, w in enumerate(wyckoff):
            why = coordination_compatible(w, d['element'], req, use_ops)
            if why:
                excluded.append(why)
                excluded_for[e].append({'label': f'{w.multiplicity}{w.letter}', 'mult': w.multiplicity, 'why': why})
            else:
                ok.add(i)
        allowed_for.append(ok)
    per_element = []
    for e, d in enumerate(demand):
        ok = allowed_for[e]
        pool = [w for k, w in enumerate(srt) if ok is None or idx[k] in ok]
        pool_idx = [i for i in idx if ok is None or i in ok]
        per_element.append([[pool_idx[k] for k in s] for s in multisets_summing_to(pool, d['count'], opts)])
    for e, d in enumerate(demand):
        if not per_element[e] and allowed_for[e] is not None and \
                multisets_summing_to(srt, d['count'], dict(opts, maxPerElement=1)):
            el = str(d['element'])
            name = el[:1].upper() + el[1:].lower()
            req = coordination[el.upper()]
            lost = [x for x in excluded_for[e] if x['mult'] <= d['count']] or excluded_for[e]
            return {'assignments': [], 'siteSymmetryExcluded': excluded, 'coordinationConflict': el,
                    'error': (f"No Wyckoff assignment gives {d['count']} {name} atoms per cell with the "
                              f"coordination stated for {name} ({req['count']} neighbour"
                              f"{'' if req['count'] == 1 else 's'}"
                              f"{', ' + req['geometry'] if req.get('geometry') else ''}). Site symmetry excludes "
                              f"{', '.join(x['label'] for x in lost)}: {lost[0]['why']}")}
        if not per_element[e]:
            avail = sorted(set(mults))
            g = 0
            for v in avail:
                g = math.gcd(g, v)
            reachable = g > 0 and d['count'] % g == 0
            min_sites = math.ceil(d['count'] / m_max)
            if reachable and min_sites > opts['maxSites']:
                why = (f"The multiplicities available ({', '.join(map(str, avail))}) can reach that total, but only "
                       f"with at least {min_sites} sites, and the search is capped at {opts['maxSites']} distinct "
                       f"site(s) per element and {opts['maxRepeat']} reuse(s) of any one position.")
            elif reachable:
                why = (f"The multiplicities available ({', '.join(map(str, avail))}) could sum to it, but not with "
                       f"these positions: one without free coordinates holds a single atom.")
            else:
                why = (f"The multiplicities available ({', '.join(map(str, avail))}) share a common factor of {g}, "
                       f"so no combination of them can sum to {d['count']}. Check Z.")
            return {'assignments': [], 'error': f"No Wyckoff assignment gives {d['count']} {d['element']} atoms per "
                                                f"cell. {why}"}
    fixed_only = {i for i, w in enumerate(wyckoff) if w.n_free == 0}
    assignments: List[dict] = []
    dropped = [0]
    cur: List[Optional[list]] = [None] * len(demand)

    def rec(e: int, used_fixed: set, used: int):
        if len(assignments) >= opts['maxTotal']:
            return
        if used > max_total_sites:
            dropped[0] += 1
            return
        if e == len(demand):
            sites = [{'element': demand[k]['element'], 'elementIdx': k, 'z': demand[k].get('z'),
                      'r': demand[k].get('r'), 'wIdx': w} for k in range(len(demand)) for w in cur[k]]
            assignments.append({'sites': sites, 'nSites': len(sites)})
            return
        for combo in per_element[e]:
            clash, added = False, []
            for w in combo:
                if w not in fixed_only:
                    continue
                if w in used_fixed:
                    clash = True
                    break
                used_fixed.add(w)
                added.append(w)
            if not clash:
                cur[e] = combo
                rec(e + 1, used_fixed, used + len(combo))
            for w in added:
                used_fixed.discard(w)
            if len(assignments) >= opts['maxTotal']:
                return

    rec(0, set(), 0)
    if not assignments and dropped[0]:
        return {'assignments': [], 'siteSymmetryExcluded': excluded, 'droppedTooManySites': dropped[0],
                'error': (f"Every Wyckoff assignment for this composition needs more than {max_total_sites} "
                          f"independent sites, which is the most the search kernel holds.")}
    if not assignments:
        clash = _fixed_point_clash(wyckoff, demand, per_element, fixed_only)
        if clash:
            return {'assignments': [], 'siteSymmetryExcluded': excluded, 'droppedTooManySites': dropped[0],
                    'fixedPointClash': True, 'error': clash}
    return {'assignments': assignments, 'truncated': len(assignments) >= opts['maxTotal'],
            'droppedTooManySites': dropped[0], 'siteSymmetryExcluded': excluded}


def normalizer_permutations(group: SpaceGroup) -> List[List[int]]:
    """Permutations of the Wyckoff positions induced by the maps x -> m x + s
    (m = +-1, s in quarter-cell steps) that normalise the group: an origin
    shift or an inversion turns an assignment into an equivalent one (the
    same |F|, the same distances).  perm[i] = the position i maps onto."""
    wyckoff = group.wyckoff
    ops = _ops(group)
    by_rot: Dict[tuple, list] = {}
    for r, t in ops:
        by_rot.setdefault(r, []).append(t)

    def close(a, b):
        return _near_int(a - b, 1e-6)

    def member(r, t):
        return any(close(u[0], t[0]) and close(u[1], t[1]) and close(u[2], t[2]) for u in by_rot.get(r, ()))

    def apply(r, t, x):
        return [r[3 * i] * x[0] + r[3 * i + 1] * x[1] + r[3 * i + 2] * x[2] + t[i] for i in range(3)]

    generic = [w.project(*_GENERIC) for w in wyckoff]
    steps = (0.0, 0.25, 0.5, 0.75)
    perms = []
    for m in (1, -1):
        for s0 in steps:
            for s1 in steps:
                for s2 in steps:
                    if m == 1 and not (s0 or s1 or s2):
                        continue
                    s = (s0, s1, s2)
                    ok = True
                    for r, w in ops:
                        Rs = [r[3 * i] * s0 + r[3 * i + 1] * s1 + r[3 * i + 2] * s2 for i in range(3)]
                        if not member(r, [m * w[i] + s[i] - Rs[i] for i in range(3)]):
                            ok = False
                            break
                    if not ok:
                        continue
                    perm = []
                    for i in range(len(wyckoff)):
                        p = generic[i]
                        q = [m * p[k] + s[k] for k in range(3)]
                        found = -1
                        for j in range(len(wyckoff)):
                            if found >= 0:
                                break
                            if wyckoff[j].multiplicity != wyckoff[i].multiplicity:
                                continue
                            for r, t in ops:
                                gq = apply(r, t, q)
                                pr = wyckoff[j].project(*gq)
                                if all(close(pr[k], gq[k]) for k in range(3)):
                                    found = j
                                    break
                        if found < 0:
                            break
                        perm.append(found)
                    if len(perm) == len(wyckoff) and any(j != i for i, j in enumerate(perm)):
                        perms.append(perm)
    return perms


def dedupe_equivalent_assignments(assignments: List[dict], group: SpaceGroup) -> dict:
    """One assignment of each set related by a normaliser permutation, the
    first met (the enumeration's order is kept)."""
    perms = normalizer_permutations(group)
    if not perms:
        return {'assignments': assignments, 'dropped': 0}

    def key_of(a, perm):
        return '|'.join(sorted(f"{s['elementIdx']}:{perm[s['wIdx']] if perm else s['wIdx']}" for s in a['sites']))
    seen, kept = set(), []
    for a in assignments:
        key = key_of(a, None)
        for perm in perms:
            k = key_of(a, perm)
            if k < key:
                key = k
        if key in seen:
            continue
        seen.add(key)
        kept.append(a)
    return {'assignments': kept, 'dropped': len(assignments) - len(kept)}


def to_search_assignment(group: SpaceGroup, assignment: dict):
    """An enumerated assignment as the search's ``wyckoff_tables.Assignment``."""
    from .wyckoff_tables import Assignment, Site
    return Assignment([Site(s['element'], s['elementIdx'], s['z'], group.wyckoff[s['wIdx']])
                       for s in assignment['sites']])


def assignment_labels(group: SpaceGroup, assignment: dict) -> List[tuple]:
    """[(element, '4c'), ...]: the form ``workloads.wyckoff_problem`` and
    ``wyckoff_tables.make_assignment`` take."""
    return [(s['element'], f"{group.wyckoff[s['wIdx']].multiplicity}{group.wyckoff[s['wIdx']].letter}")
            for s in assignment['sites']]
