"""Wyckoff assignments consistent with a composition: which (element,
Wyckoff position) sets the device searches.

Behaviour follows the reference's assignment step (js/wyckoff_assign.js:184-754:
the per-element position multisets, the site-symmetry exclusions for a stated
coordination, the combination with no fixed point shared by two elements and
at most 32 sites, failure messages that name the constraint, and the removal
of assignments that an origin shift or an inversion of the group maps onto
one another), pinned by its regression counts.  The construction is this
module's own:

* per element, the position multisets summing to the count are the
  solutions of a bounded knapsack over the multiplicities (a position without
  free coordinates at most once, a free one up to ``maxRepeat`` times).  A
  reachability table, built backwards over the positions, holds for every
  remainder the bitmask of site counts that can still complete it; the
  solutions are then read off site count by site count (fewest sites first),
  expanding only branches the table says complete;
* elements are combined by a breadth-first fold over states (bitmask of the
  fixed points taken, sites used): a choice joins a state when its own
  fixed-point mask is disjoint from the state's;
* a site's symmetry is read from the operators that fix a generic point of
  its subspace, all operators at once in integer arithmetic over 1/24;
* equivalent assignments are found through the group's affine normaliser
  x -> m x + s (m = +-1): every shift s at the group's own translation
  resolution (1/24) that conjugates the group onto itself, reduced to cosets
  of the group with ``SymOp.compose``; each coset permutes the positions,
  found by an exact subspace test of the mapped generic point.

Positions are the group's ``wyckoff`` list; ``demand`` is
[{'element', 'count' (atoms per cell), 'z', 'r'}].
"""
from __future__ import annotations

import math
from fractions import Fraction
from itertools import product
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .symmetry import IDENT, INV, TDEN, SpaceGroup, SymOp, WyckoffPosition

MAX_SITES = 32            # sites one assignment may hold (the search kernel's limit)
MAX_ASSIGNMENTS = 4000    # enumeration cap

# Coordination polyhedra without an inversion centre.
NON_CENTROSYMMETRIC_GEOMETRY = {'tetrahedral', 'trigonal-planar', 'trigonal-pyramidal', 'square-pyramidal',
                                'trigonal-prismatic', 'see-saw', 'bent'}

# Central atoms for which four neighbours mean a tetrahedron (oxoanion and
# framework formers; four-coordinate d8 cations and O are often square planar).
TETRAHEDRAL_AT_FOUR = {'B', 'C', 'N', 'F', 'AL', 'SI', 'P', 'S', 'CL', 'GA', 'GE', 'AS', 'SE', 'BR', 'V', 'CR', 'MN',
                       'FE', 'CO', 'ZN', 'MO', 'W', 'TC', 'RE', 'BE', 'I', 'XE'}

# A point no special position passes through: each coordinate a fraction of
# 24 * 1009, so operators (translations in 1/24) act on it in integers.
_SCALE = TDEN * 1009
_GEN = (137, 251, 409)


def _label(w: WyckoffPosition) -> str:
    return f'{w.multiplicity}{w.letter}'


def _generic_point(w: WyckoffPosition) -> Tuple[Fraction, Fraction, Fraction]:
    g = [Fraction(v, 1009) for v in _GEN]
    return tuple(sum(w.P[3 * i + k] * g[k] for k in range(3)) + w.T[i] for i in range(3))


# ---------------------------------------------------------------------------
# Site symmetry
# ---------------------------------------------------------------------------
def _op_arrays(ops: Sequence) -> Tuple[np.ndarray, np.ndarray]:
    """Rotations (n, 3, 3) and translations in 1/24 (n, 3) of SymOps or (r, t_frac) pairs."""
    R, T = [], []
    for o in ops:
        if isinstance(o, SymOp):
            R.append(o.r)
            T.append(o.t)
        else:
            r, t = o
            R.append(tuple(r))
            T.append(tuple(int(round(v * TDEN)) for v in t))
    return np.array(R, dtype=np.int64).reshape(-1, 3, 3), np.array(T, dtype=np.int64).reshape(-1, 3)


def site_rotations(w: WyckoffPosition, ops: Sequence) -> List[Tuple[int, ...]]:
    """Rotation parts of the operators fixing a generic point of ``w`` modulo
    the lattice (exact: the point is held in units of 1 / (24 * 1009))."""
    R, T = _op_arrays(ops)
    p = np.array([int(v * _SCALE) for v in _generic_point(w)], dtype=np.int64)
    img = np.einsum('nij,j->ni', R, p) + T * (_SCALE // TDEN)
    fixed = np.all((img - p) % _SCALE == 0, axis=1)
    return [tuple(int(v) for v in R[k].reshape(-1)) for k in np.nonzero(fixed)[0]]


def site_has_inversion(w: WyckoffPosition, ops: Sequence) -> bool:
    return INV in site_rotations(w, ops)


def coordination_compatible(w: WyckoffPosition, element: str, req: Optional[dict], ops) -> Optional[str]:
    """None when an atom of ``element`` with coordination ``req`` ({'count',
    'geometry'}) may sit on ``w``; otherwise why not.  A site on an inversion
    centre sees its neighbours in antipodal pairs, so it needs an even
    count, and no polyhedron lacking a centre of symmetry (stated, or the
    tetrahedron implied by four neighbours of a tetrahedral former) fits it."""
    if not req or not req.get('count') or req['count'] <= 0 or not ops:
        return None
    if not site_has_inversion(w, ops):
        return None
    n = int(req['count'])
    if n % 2:
        return (f"{w.multiplicity}{w.letter} is an inversion centre, where neighbours come in opposite pairs; "
                f"{element} with {n} neighbours (an odd number) cannot sit there.")
    geom = str(req['geometry']).lower() if req.get('geometry') else None
    if not geom and n == 4 and str(element).upper() in TETRAHEDRAL_AT_FOUR:
        geom = 'tetrahedral'
    if geom in NON_CENTROSYMMETRIC_GEOMETRY:
        return (f"{w.multiplicity}{w.letter} is an inversion centre, and a {geom} arrangement around {element} "
                f"has no centre of symmetry to put there.")
    return None


# ---------------------------------------------------------------------------
# Position multisets per element: bounded knapsack with a reachability table
# ---------------------------------------------------------------------------
def multisets_summing_to(positions: Sequence[WyckoffPosition], target: int, opts: dict) -> List[List[int]]:
    """Index multisets of ``positions`` whose multiplicities sum to
    ``target``, each index at most once for a position without free
    coordinates and at most ``maxRepeat`` times otherwise, with at most
    ``maxSites`` sites; at most ``maxPerElement`` of them, fewest sites first,
    then in order of the positions (indices non-decreasing within one)."""
    n = len(positions)
    max_sites = int(opts['maxSites'])
    limit = int(opts['maxPerElement'])
    mult = [int(p.multiplicity) for p in positions]
    cap = [0 if m <= 0 else (1 if p.n_free == 0 else int(opts['maxRepeat'])) for p, m in zip(positions, mult)]
    # reach[i][r]: bit k set when positions i.. can make remainder r with exactly k sites
    reach = [[0] * (target + 1) for _ in range(n + 1)]
    reach[n][0] = 1
    for i in range(n - 1, -1, -1):
        nxt, cur = reach[i + 1], reach[i]
        for r in range(target + 1):
            bits = 0
            for c in range(0, cap[i] + 1):
                if c * mult[i] > r:
                    break
                bits |= nxt[r - c * mult[i]] << c
            cur[r] = bits & ((1 << (max_sites + 1)) - 1)
    out: List[List[int]] = []
    counts = [0] * n

    def walk(i: int, r: int, k: int):
        """Positions i.., remainder r, exactly k more sites."""
        if len(out) >= limit:
            return
        if i == n:
            out.append([j for j in range(n) for _ in range(counts[j])])
            return
        for c in range(min(cap[i], k), -1, -1):
            rest = r - c * mult[i]
            if rest < 0 or not (reach[i + 1][rest] >> (k - c)) & 1:
                continue
            counts[i] = c
            walk(i + 1, rest, k - c)
            counts[i] = 0

    for k in range(1, max_sites + 1):
        if (reach[0][target] >> k) & 1:
            walk(0, target, k)
        if len(out) >= limit:
            break
    return out


# ---------------------------------------------------------------------------
# Enumeration
# ---------------------------------------------------------------------------
def _join(words: Sequence[str]) -> str:
    return words[0] if len(words) == 1 else ', '.join(words[:-1]) + ' and ' + words[-1]


def _no_multiset_reason(d: dict, mults: Sequence[int], m_max: int, opts: dict) -> str:
    avail = sorted(set(mults))
    g = 0
    for v in avail:
        g = math.gcd(g, v)
    shown = ', '.join(map(str, avail))
    if g == 0 or d['count'] % g:
        return (f"Every available multiplicity ({shown}) is a multiple of {g}, a common factor that "
                f"{d['count']} does not share, so no combination reaches it. Check Z.")
    need = math.ceil(d['count'] / m_max)
    if need > opts['maxSites']:
        return (f"The multiplicities ({shown}) reach {d['count']} only with {need} or more sites; the search "
                f"takes at most {opts['maxSites']} sites per element and {opts['maxRepeat']} uses of one "
                f"position.")
    return (f"The multiplicities ({shown}) could add up to it, but the positions without free coordinates "
            f"hold one atom each, and those available do not suffice.")


def enumerate_assignments(group: SpaceGroup, demand: Sequence[dict], options: Optional[dict] = None) -> dict:
    """Every assignment of Wyckoff positions to the demanded atoms per cell.

    Returns {'assignments': [{'sites': [{'element', 'elementIdx', 'z', 'r',
    'wIdx'}], 'nSites'}], 'truncated', 'droppedTooManySites',
    'siteSymmetryExcluded'}; when none exists the list is empty and 'error'
    says which constraint left nothing."""
    options = dict(options or {})
    wyckoff = group.wyckoff
    ceiling = options.get('ceiling', 24)
    mults = [w.multiplicity for w in wyckoff if w.multiplicity > 0]
    m_max = max(mults) if mults else 1
    need = min(ceiling, math.ceil(max((d['count'] for d in demand), default=0) / m_max))
    opts = {'maxSites': min(ceiling, max(options.get('maxSites', 4), need)),
            'maxRepeat': min(ceiling, max(options.get('maxRepeat', 4), need)),
            'maxPerElement': options.get('maxPerElement', 500),
            'maxTotal': options.get('maxTotal', MAX_ASSIGNMENTS)}
    max_total_sites = options.get('maxTotalSites', MAX_SITES)
    coordination = options.get('coordination') or {}
    check_symmetry = options.get('symOps', True)
    order = sorted(range(len(wyckoff)), key=lambda i: (-wyckoff[i].multiplicity, i))
    excluded: List[str] = []
    per_element: List[List[List[int]]] = []
    for e, d in enumerate(demand):
        req = coordination.get(str(d['element']).upper())
        allowed, lost = order, []
        if req and check_symmetry:
            allowed = []
            for i in order:
                why = coordination_compatible(wyckoff[i], d['element'], req, group.ops)
                if why:
                    excluded.append(why)
                    lost.append((wyckoff[i], why))
                else:
                    allowed.append(i)
        sets = [[allowed[k] for k in s]
                for s in multisets_summing_to([wyckoff[i] for i in allowed], d['count'], opts)]
        if not sets:
            name = str(d['element'])[:1].upper() + str(d['element'])[1:].lower()
            if lost and multisets_summing_to([wyckoff[i] for i in order], d['count'], dict(opts, maxPerElement=1)):
                fits = [x for x in lost if x[0].multiplicity <= d['count']] or lost
                geom = f", {req['geometry']}" if req.get('geometry') else ''
                return {'assignments': [], 'siteSymmetryExcluded': excluded, 'coordinationConflict': d['element'],
                        'error': (f"{d['count']} {name} atoms per cell cannot be placed with the coordination "
                                  f"stated for {name} ({req['count']} neighbours{geom}): "
                                  f"{_join([_label(w) for w, _ in fits])} would be needed, and {fits[0][1]}")}
            return {'assignments': [], 'error': f"No Wyckoff assignment gives {d['count']} {d['element']} atoms "
                                                f"per cell. {_no_multiset_reason(d, mults, m_max, opts)}"}
        per_element.append(sets)

    # breadth-first fold over (fixed points taken, sites used)
    fixed_bit = {i: 1 << k for k, i in enumerate(i for i, w in enumerate(wyckoff) if w.n_free == 0)}
    choice_mask = [[sum(fixed_bit.get(i, 0) for i in s) for s in sets] for sets in per_element]
    states: List[Tuple[int, int, Tuple[int, ...]]] = [(0, 0, ())]
    dropped = truncated = 0
    for e, sets in enumerate(per_element):
        grown = []
        for mask, used, picks in states:
            for j, s in enumerate(sets):
                if mask & choice_mask[e][j]:
                    continue
                if used + len(s) > max_total_sites:
                    dropped += 1
                    continue
                grown.append((mask | choice_mask[e][j], used + len(s), picks + (j,)))
                if len(grown) >= opts['maxTotal']:
                    truncated = 1
                    break
            if len(grown) >= opts['maxTotal']:
                break
        states = grown
    assignments = []
    for _, used, picks in states:
        sites = [{'element': demand[e]['element'], 'elementIdx': e, 'z': demand[e].get('z'),
                  'r': demand[e].get('r'), 'wIdx': i} for e, j in enumerate(picks) for i in per_element[e][j]]
        assignments.append({'sites': sites, 'nSites': used})
    if not assignments:
        err = None
        if dropped:
            err = (f"Every Wyckoff assignment for this composition needs more than {max_total_sites} independent "
                   f"sites, more than the search kernel holds.")
        else:
            # elements that can only go on fixed points, competing for them
            bound = [e for e, masks in enumerate(choice_mask) if all(masks)]
            pool = sorted({i for e in bound for s in per_element[e] for i in s if i in fixed_bit})
            if len(bound) >= 2:
                who = [f"{demand[e]['element']} ({demand[e]['count']} per cell)" for e in bound]
                err = (f"{_join(who)} fit only on positions without free coordinates "
                       f"({_join([_label(wyckoff[i]) for i in pool])}), and a fixed point holds one element, so "
                       f"no assignment gives each of them its own sites. The search builds ordered models, one "
                       f"element per site.")
        out = {'assignments': [], 'siteSymmetryExcluded': excluded, 'droppedTooManySites': dropped}
        if err:
            out['error'] = err
            out['fixedPointClash'] = not dropped
        return out
    return {'assignments': assignments, 'truncated': bool(truncated), 'droppedTooManySites': dropped,
            'siteSymmetryExcluded': excluded}


# ---------------------------------------------------------------------------
# Equivalent assignments: the affine normaliser x -> m x + s
# ---------------------------------------------------------------------------
def normalizer_cosets(group: SpaceGroup) -> List[SymOp]:
    """Representatives, other than the group's own, of the cosets of the
    group in its normaliser among the maps x -> m x + s (m = +-1, s in
    1/24): those for which (R, m t + (I - R) s) belongs to the group for
    every (R, t) in it.  Each maps structures onto equivalent ones (the same
    |F|, the same distances)."""
    R, T = _op_arrays(group.ops)
    # membership table: rotation id x translation code (t0 * 576 + t1 * 24 + t2)
    rot_ids: Dict[Tuple[int, ...], int] = {}
    rid = np.array([rot_ids.setdefault(tuple(int(v) for v in R[k].reshape(-1)), len(rot_ids))
                    for k in range(len(R))], dtype=np.int64)
    table = np.zeros((len(rot_ids), TDEN ** 3), dtype=bool)
    table[rid, (T[:, 0] % TDEN) * TDEN * TDEN + (T[:, 1] % TDEN) * TDEN + T[:, 2] % TDEN] = True
    I3 = np.eye(3, dtype=np.int64)
    shifts = np.array(list(product(range(TDEN), repeat=3)), dtype=np.int64)         # (24^3, 3)
    found: List[SymOp] = []
    for m in (1, -1):
        # conjugate translations of every operator for every shift: (shifts, ops, 3)
        conj = (m * T[None, :, :] + np.einsum('nij,sj->sni', I3[None] - R, shifts)) % TDEN
        code = conj[..., 0] * TDEN * TDEN + conj[..., 1] * TDEN + conj[..., 2]
        ok = table[rid[None, :], code].all(axis=1)
        mat = IDENT if m == 1 else INV
        for s in shifts[ok]:
            found.append(SymOp(mat, tuple(int(v) for v in s)))
    # cosets N G: keyed by their least element; the group's own coset is dropped
    def canon(o: SymOp):
        return (o.r, tuple(v % TDEN for v in o.t))
    own = min(canon(g) for g in group.ops)
    reps: Dict[tuple, SymOp] = {}
    for n in found:
        k = min(canon(n.compose(g)) for g in group.ops)
        if k != own and k not in reps:
            reps[k] = n
    return list(reps.values())


def _on_subspace(w: WyckoffPosition, y: Sequence[Fraction]) -> bool:
    return all(sum(w.P[3 * i + k] * y[k] for k in range(3)) + w.T[i] == y[i] for i in range(3))


def _position_of(group: SpaceGroup, q: Sequence[Fraction], mult: int) -> int:
    """The position (of multiplicity ``mult``) whose orbit holds the point q."""
    images = []
    for o in group.ops:
        y = [sum(o.r[3 * i + k] * q[k] for k in range(3)) + Fraction(o.t[i], TDEN) for i in range(3)]
        images.append([v - math.floor(v) for v in y])
    for j, w in enumerate(group.wyckoff):
        if w.multiplicity != mult:
            continue
        for y in images:
            for n in product((-1, 0, 1), repeat=3):
                if _on_subspace(w, [y[i] + n[i] for i in range(3)]):
                    return j
    return -1


def normalizer_permutations(group: SpaceGroup) -> List[List[int]]:
    """For each normaliser coset that moves some position, perm[i] = the
    position that position i maps onto."""
    perms = []
    if len(group.wyckoff) < 2:
        return perms
    generic = [_generic_point(w) for w in group.wyckoff]
    for n in normalizer_cosets(group):
        perm = []
        for i, w in enumerate(group.wyckoff):
            p = generic[i]
            q = [n.r[4 * k] * p[k] + Fraction(n.t[k], TDEN) for k in range(3)]
            j = _position_of(group, q, w.multiplicity)
            if j < 0:
                break
            perm.append(j)
        if len(perm) == len(group.wyckoff) and perm != list(range(len(perm))):
            perms.append(perm)
    return perms


def dedupe_equivalent_assignments(assignments: List[dict], group: SpaceGroup) -> dict:
    """The first assignment met of each class related by a normaliser
    permutation (the enumeration's order is kept)."""
    perms = normalizer_permutations(group)
    if not perms:
        return {'assignments': list(assignments), 'dropped': 0}

    def canonical(a):
        base = [(s['elementIdx'], s['wIdx']) for s in a['sites']]
        return min([tuple(sorted(base))] + [tuple(sorted((e, p[i]) for e, i in base)) for p in perms])
    seen, kept = set(), []
    for a in assignments:
        c = canonical(a)
        if c not in seen:
            seen.add(c)
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
    return [(s['element'], _label(group.wyckoff[s['wIdx']])) for s in assignment['sites']]
