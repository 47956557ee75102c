"""Packed tables the Wyckoff trial kernel reads.

* ``build_assignment_tables`` follows js/wyckoff_assign.js:756-944: per
  assignment and generated atom, ``genPack = site | op << 8 | type << 20 |
  skip << 24`` (skip marks a centring translate of an earlier image of the same
  site, left out of the |F|^2 sums), and per (assignment, site) the projector
  ``siteProj`` = P(9), T(3), zero for unused site slots.
* ``build_restraint_tables`` follows js/wyckoff_assign.js:954-1133: the float
  table [z by type | rMin (nElem x nElem) | rules (7 floats each: aType, bType,
  dmin, dmax, count, mode, geometry)].
* ``pack_sym_ops`` follows js/wyckoff_assign.js:1134-1139 (12 floats per
  operator, r then t).
* ``project_sites`` follows js/wyckoff_assign.js:1155-1187.

Capacities are the reference kernel's (js/wyckoff_assign.js:60-70 and
js/wyckoff_limits.js:10-62): at most 32 sites per assignment, 8 elements,
4096 operators, 32 rules and 256 neighbour slots.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from .symmetry import IDENT, SpaceGroup, SymOp, WyckoffPosition

WY_MAX_SITES = 32
WY_MAX_ELEM = 8
WY_MAX_OPS = 4096
WY_MAX_RULES = 32
WY_MAX_COORD_SLOTS = 256
WY_BASE_RULES = 8
WY_BASE_COORD_SLOTS = 64
GEOMETRIES = {'linear': (1, 2), 'trigonal-planar': (2, 3), 'tetrahedral': (3, 4),
              'square-planar': (4, 4), 'octahedral': (5, 6)}
_GEOM_WORDS = {'linear': 'linear', 'triangle': 'trigonal-planar', 'triangular': 'trigonal-planar',
               'trigonal': 'trigonal-planar', 'trigonal-planar': 'trigonal-planar',
               'tetrahedron': 'tetrahedral', 'tetrahedral': 'tetrahedral', 'tetra': 'tetrahedral',
               'square': 'square-planar', 'square-planar': 'square-planar', 'planar': 'square-planar',
               'octahedron': 'octahedral', 'octahedral': 'octahedral', 'octa': 'octahedral'}


@dataclass
class Site:
    element: str
    element_idx: int
    z: float
    w: WyckoffPosition


@dataclass
class Assignment:
    sites: List[Site]

    @property
    def n_sites(self) -> int:
        return len(self.sites)


def make_assignment(group: SpaceGroup, demand: Sequence[dict], labels: Sequence[tuple]) -> Assignment:
    """[('Pb', '4c'), ('S', '4c'), ...] -> Assignment, element indices from ``demand`` order."""
    idx = {d['element'].upper(): i for i, d in enumerate(demand)}
    sites = []
    for el, pos in labels:
        i = idx[el.upper()]
        sites.append(Site(el, i, demand[i]['z'], group.position(pos)))
    return Assignment(sites)


@dataclass
class AssignmentTables:
    n_tot: int
    max_sites: int
    gen_site: np.ndarray
    gen_op: np.ndarray
    gen_type: np.ndarray
    gen_skip: np.ndarray
    gen_pack: np.ndarray
    site_proj: np.ndarray        # float32 (nA * maxSites * 12)
    site_count: np.ndarray
    centring: List[tuple]
    warnings: List[str] = field(default_factory=list)


_SS_GENERIC = (0.1234567, 0.3456789, 0.5678901)


def build_assignment_tables(assignments: Sequence[Assignment], group: SpaceGroup,
                            demand: Sequence[dict]) -> AssignmentTables:
    ops = group.ops
    n_tot = sum(d['count'] for d in demand)
    centring = []
    for o in ops:
        if o.r == IDENT:
            c = [v - math.floor(v + 1e-9) for v in o.t_frac]
            if any(abs(v) > 1e-6 and abs(v - 1) > 1e-6 for v in c):
                centring.append(tuple(c))

    def near0(v):
        return abs(v - round(v)) < 1e-4

    nA = len(assignments)
    max_sites = max((A.n_sites for A in assignments), default=0)
    if max_sites > WY_MAX_SITES:
        raise ValueError(f'The widest assignment needs {max_sites} independent Wyckoff sites; '
                         f'the search kernel holds {WY_MAX_SITES}.')
    if len(demand) > WY_MAX_ELEM:
        raise ValueError(f'{len(demand)} distinct elements; the search kernel holds {WY_MAX_ELEM}.')
    if len(ops) > WY_MAX_OPS:
        raise ValueError(f'{len(ops)} symmetry operators; genOp is packed 12 bits wide.')
    gen_site = np.zeros(nA * n_tot, dtype=np.uint32)
    gen_op = np.zeros(nA * n_tot, dtype=np.uint32)
    gen_type = np.zeros(nA * n_tot, dtype=np.uint32)
    gen_skip = np.zeros(nA * n_tot, dtype=np.uint8)
    site_proj = np.zeros(nA * max_sites * 12, dtype=np.float32)
    site_count = np.zeros(nA, dtype=np.uint32)
    warnings = []
    for ai, A in enumerate(assignments):
        g = 0
        for si, s in enumerate(A.sites):
            cos = s.w.coset_ops
            p = s.w.project(*_SS_GENERIC) if centring else None
            seen = []
            for op in cos:
                if g >= n_tot:
                    break
                gen_site[ai * n_tot + g] = si
                gen_op[ai * n_tot + g] = op
                gen_type[ai * n_tot + g] = s.element_idx
                if p is not None:
                    O = ops[op]
                    r, t = O.r, O.t_frac
                    q = [r[3 * i] * p[0] + r[3 * i + 1] * p[1] + r[3 * i + 2] * p[2] + t[i] for i in range(3)]
                    if any(all(near0(q[i] - e[i] - c[i]) for i in range(3)) for e in seen for c in centring):
                        gen_skip[ai * n_tot + g] = 1
                    seen.append(q)
                g += 1
            b = (ai * max_sites + si) * 12
            site_proj[b:b + 9] = s.w.P_float
            site_proj[b + 9:b + 12] = s.w.T_float
        site_count[ai] = A.n_sites
        if g != n_tot:
            warnings.append(f'Assignment {ai} generated {g} atoms, expected {n_tot}.')
    n_cent = len(centring) + 1
    use_centring = n_cent > 1 and n_tot % n_cent == 0
    for ai in range(nA):
        if not use_centring:
            break
        kept = int((gen_skip[ai * n_tot:(ai + 1) * n_tot] == 0).sum())
        if kept != n_tot // n_cent:
            use_centring = False
    if n_cent > 1 and not use_centring:
        warnings.append('The orbits do not split into centring classes as expected; the structure factors sum over the whole cell.')
        gen_skip[:] = 0
    gen_pack = (gen_site | (gen_op << 8) | (gen_type << 20) | (gen_skip.astype(np.uint32) << 24)).astype(np.uint32)
    return AssignmentTables(n_tot, max_sites, gen_site, gen_op, gen_type, gen_skip, gen_pack, site_proj,
                            site_count, centring if use_centring else [], warnings)


@dataclass
class RestraintTables:
    tables: np.ndarray        # float32 [zByType | rMin | rules]
    r_min_off: int
    rule_off: int
    n_rules: int
    n_elem: int
    slots_needed: int
    geometry: bool
    max_distance: float
    rules: List[list]
    problems: List[str]


def build_restraint_tables(demand: Sequence[dict], windows: Sequence[dict] = (),
                           min_contact: Optional[float] = None) -> RestraintTables:
    n_elem = len(demand)
    idx = {d['element'].upper(): i for i, d in enumerate(demand)}
    floor_ = 1.0 if min_contact is None else (min_contact if (math.isfinite(min_contact) and min_contact > 0) else 0.0)
    z_by_type = [d['z'] for d in demand]
    r_min = np.full(n_elem * n_elem, floor_, dtype=np.float64)
    problems, rules = [], []
    for w in windows:
        a = idx.get(str(w['a']).upper())
        b = idx.get(str(w['b']).upper())
        if a is None or b is None:
            problems.append(f"Constraint {w['a']}-{w['b']} names an element that is not in the composition.")
            continue
        dmin = w.get('dmin')
        dmax = w.get('dmax')
        dmin = float(dmin) if dmin is not None and math.isfinite(dmin) else None
        dmax = float(dmax) if dmax is not None and math.isfinite(dmax) else None
        if dmin is not None and dmax is not None and dmax < dmin:
            problems.append(f"Constraint {w['a']}-{w['b']} has dmax ({dmax}) below dmin ({dmin}).")
            continue
        if dmin is not None:
            r_min[a * n_elem + b] = dmin
            r_min[b * n_elem + a] = dmin
        cnt = w.get('count')
        has_count = cnt is not None and math.isfinite(cnt) and cnt >= 0
        mode = (2 if w.get('countMode') == 'atleast' else 1) if has_count else 0
        if not has_count and dmax is None:
            continue
        geom_name = _GEOM_WORDS.get(str(w.get('geometry')).lower()) if w.get('geometry') else None
        if w.get('geometry') and geom_name is None:
            problems.append(f"Constraint {w['a']}-{w['b']}: unknown geometry \"{w['geometry']}\" was ignored.")
        geom = GEOMETRIES.get(geom_name) if geom_name else None
        if geom and (not has_count or cnt != geom[1] or dmax is None):
            raise ValueError(f"Constraint {w['a']}-{w['b']}: a {w['geometry']} needs exactly {geom[1]} "
                             f"neighbours and an upper distance.")
        rec = [a, b, dmin if dmin is not None else 0.0, dmax if dmax is not None else math.inf,
               cnt if has_count else 0, mode, geom[0] if geom else 0]
        rules.append(rec)
        if not has_count and w.get('bothWays', True) is not False and a != b:
            rules.append([b, a, dmin if dmin is not None else 0.0, dmax if dmax is not None else math.inf,
                          0, 0, 0])
    if len(rules) > WY_MAX_RULES:
        raise ValueError(f'{len(rules)} distance rules; the search kernel holds {WY_MAX_RULES}.')
    slots = sum(r[4] for r in rules if r[5] != 0)
    if slots > WY_MAX_COORD_SLOTS:
        raise ValueError(f'The coordination numbers add up to {slots} neighbour slots; the kernel tracks '
                         f'{WY_MAX_COORD_SLOTS}.')
    r_min_off = len(z_by_type)
    rule_off = r_min_off + len(r_min)
    tables = np.zeros(rule_off + 7 * len(rules), dtype=np.float32)
    tables[:r_min_off] = z_by_type
    tables[r_min_off:rule_off] = r_min
    for k, r in enumerate(rules):
        tables[rule_off + 7 * k: rule_off + 7 * k + 7] = r
    maxd = float(r_min.max()) if len(r_min) else 0.0
    for r in rules:
        if math.isfinite(r[3]):
            maxd = max(maxd, r[3])
    return RestraintTables(tables, r_min_off, rule_off, len(rules), n_elem, slots,
                           any(r[6] > 0 for r in rules), maxd, rules, problems)


def pack_sym_ops(ops: Sequence[SymOp]) -> np.ndarray:
    out = np.zeros(len(ops) * 12, dtype=np.float32)
    for i, o in enumerate(ops):
        out[i * 12:i * 12 + 9] = o.r
        out[i * 12 + 9:i * 12 + 12] = o.t_frac
    return out


def project_sites(positions: np.ndarray, particle: int, assign: int, T: AssignmentTables) -> None:
    """Project one particle's coordinates onto its assignment's subspaces, in place."""
    nS = int(T.site_count[assign])
    stride = T.max_sites * 3
    sp = T.site_proj.astype(np.float64)
    for s in range(nS):
        b = (assign * T.max_sites + s) * 12
        o = particle * stride + s * 3
        x, y, z = (float(positions[o + i]) for i in range(3))
        for i in range(3):
            v = sp[b + 3 * i] * x + sp[b + 3 * i + 1] * y + sp[b + 3 * i + 2] * z + sp[b + 9 + i]
            positions[o + i] = v - math.floor(v)
    for s in range(nS, T.max_sites):
        o = particle * stride + s * 3
        positions[o:o + 3] = 0


def wyckoff_freedom(w: WyckoffPosition) -> int:
    return w.n_free
