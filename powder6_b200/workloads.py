"""Seeded synthetic problems with the shapes of the benchmark configurations.

The reference measures no public dataset for this path; these generators stand
in for real extracted intensities with the stated cells, sites, resolution and
noise.

* ``wyckoff_problem``: a Wyckoff search problem.  Default: Pnma, a = 8.48,
  b = 5.40, c = 6.96 A, sites Pb 4c, S 4c, O 4c, O 4c, O 8d (PbSO4-like),
  seeded random true coordinates, |F|^2 of every unique reflection to
  d_min = 1.2 A with X-ray f(s) (Waasmaier-Kirfel) and overall B = 0, 2 %
  Gaussian noise and sigma = 2 % of the noiseless value.
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .crystal import inverse3, orth_matrix, reduced_cell
from .reflections import (PackedReflections, gaussian_form_factor, generate_reflections, pack_reflections,
                          scattering_table)
from .symmetry import SpaceGroup, has_inversion_at_origin, space_group
from .wyckoff_tables import (Assignment, AssignmentTables, RestraintTables, build_assignment_tables,
                             build_restraint_tables, make_assignment, pack_sym_ops)

DATA = Path(__file__).resolve().parent / 'data'


def load_form_factor_table() -> Dict[str, dict]:
    return json.loads((DATA / 'xray_wk1995_subset.json').read_text())['table']


def mulberry32(seed: int):
    """The reference's seeded host stream (js/swarm_wyckoff.js:354-363)."""
    s = seed & 0xFFFFFFFF

    def rnd():
        nonlocal s
        s = (s + 0x6D2B79F5) & 0xFFFFFFFF
        t = s
        t = ((t ^ (t >> 15)) * (t | 1)) & 0xFFFFFFFF
        t ^= (t + ((t ^ (t >> 7)) * (t | 61) & 0xFFFFFFFF)) & 0xFFFFFFFF
        return ((t ^ (t >> 14)) & 0xFFFFFFFF) / 4294967296.0
    return rnd


@dataclass
class WyckoffProblem:
    group: SpaceGroup
    cell: Dict[str, float]
    demand: List[dict]
    assignments: List[Assignment]
    tables: AssignmentTables
    refl: PackedReflections
    f_tab: np.ndarray
    n_elem: int
    restraints: RestraintTables
    sym_packed: np.ndarray
    centro: bool
    orth: np.ndarray
    xform: np.ndarray
    inv_orth: np.ndarray
    min_image_shell: int
    true_coords: Optional[np.ndarray] = None
    rows: List[dict] = field(default_factory=list)
    pen_clash: float = 0.05
    pen_bond: float = 0.10
    pen_coord: float = 0.03
    pen_geom: float = 1.0

    @property
    def n_tot(self) -> int:
        return self.tables.n_tot

    @property
    def max_sites(self) -> int:
        return self.tables.max_sites


def structure_factors_fp64(group: SpaceGroup, assignment: Assignment, coords: np.ndarray,
                           hkl: np.ndarray, f_of: np.ndarray) -> np.ndarray:
    """|F|^2 of the full cell (every image, both sine and cosine), FP64.
    hkl (n, 3) ints; f_of (n, nElem) scattering factors per reflection."""
    F = np.zeros(len(hkl), dtype=np.complex128)
    h = hkl.astype(np.float64)
    for si, s in enumerate(assignment.sites):
        p = s.w.project(*coords[si * 3:si * 3 + 3])
        for oi in s.w.coset_ops:
            o = group.ops[oi]
            x = np.array([sum(o.r[3 * i + k] * p[k] for k in range(3)) + o.t_frac[i] for i in range(3)])
            x -= np.floor(x)
            F += f_of[:, s.element_idx] * np.exp(2j * np.pi * (h @ x))
    return np.abs(F) ** 2


def _min_contact(group: SpaceGroup, assignment: Assignment, coords: np.ndarray, red) -> float:
    """Shortest nearest-image distance between any two atoms of the generated cell."""
    pts = []
    for si, s in enumerate(assignment.sites):
        p = s.w.project(*coords[si * 3:si * 3 + 3])
        for oi in s.w.coset_ops:
            o = group.ops[oi]
            pts.append([sum(o.r[3 * i + k] * p[k] for k in range(3)) + o.t_frac[i] for i in range(3)])
    x = np.array(pts) % 1.0
    d = x[:, None, :] - x[None, :, :]
    q = np.einsum('ij,abj->abi', red.xform.reshape(3, 3), d)
    q -= np.round(q)
    c = np.einsum('ij,abj->abi', red.orth.reshape(3, 3), q)
    r = np.sqrt((c ** 2).sum(-1))
    np.fill_diagonal(r, np.inf)
    return float(r.min()) if len(x) > 1 else np.inf


def wyckoff_problem(seed: int = 1, group_number: int = 62,
                    cell: Optional[Dict[str, float]] = None,
                    composition: Sequence[Tuple[str, int]] = (('Pb', 4), ('S', 4), ('O', 16)),
                    sites: Sequence[Tuple[str, str]] = (('Pb', '4c'), ('S', '4c'), ('O', '4c'), ('O', '4c'),
                                                        ('O', '8d')),
                    dmin: float = 1.2, wavelength: float = 1.5406, noise: float = 0.02,
                    windows: Sequence[dict] = (), min_contact: Optional[float] = None,
                    extra_assignments: Sequence[Sequence[Tuple[str, str]]] = (),
                    true_min_contact: float = 1.6, contact_attempts: int = 2000) -> WyckoffProblem:
    cell = dict(cell or {'a': 8.48, 'b': 5.40, 'c': 6.96, 'alpha': 90.0, 'beta': 90.0, 'gamma': 90.0})
    group = space_group(group_number)
    ff_table = load_form_factor_table()
    demand = [{'element': el, 'count': n, 'z': ff_table[el]['Z'] if el in ff_table else 1} for el, n in composition]
    assignment = make_assignment(group, demand, sites)
    assignments = [assignment] + [make_assignment(group, demand, a) for a in extra_assignments]
    tables = build_assignment_tables(assignments, group, demand)
    rng = np.random.default_rng(seed)
    red0 = reduced_cell(cell)
    true = np.zeros(tables.max_sites * 3)
    for _attempt in range(contact_attempts):
        for si, s in enumerate(assignment.sites):
            true[si * 3:si * 3 + 3] = np.array(s.w.project(*rng.random(3))) % 1.0
        if _min_contact(group, assignment, true, red0) >= true_min_contact:
            break
    refs = generate_reflections(cell, group.ops, dmin, with_eq=False)
    if tables.centring:
        refs = [r for r in refs if all(abs((r.h * c[0] + r.k * c[1] + r.l * c[2]) -
                                           round(r.h * c[0] + r.k * c[1] + r.l * c[2])) < 1e-6
                                       for c in tables.centring)]
    hkl = np.array([[r.h, r.k, r.l] for r in refs], dtype=np.int64)
    ff = gaussian_form_factor(ff_table)
    s_arr = np.array([1.0 / r.d0 for r in refs])
    f_of = np.array([[ff(d['element'], s) for d in demand] for s in s_arr])
    I = structure_factors_fp64(group, assignment, true, hkl, f_of)
    floor_ = 1e-3 * float(np.mean(I)) if len(I) else 1.0
    rows = []
    for r, i_true in zip(refs, I):
        sigma = noise * max(i_true, floor_)
        fo2 = i_true + rng.normal() * sigma
        tth = 2 * math.degrees(math.asin(min(1.0, wavelength / (2 * r.d0))))
        rows.append({'h': r.h, 'k': r.k, 'l': r.l, 'mult': r.m, 'Fo2': fo2, 'sigma': sigma, 'd': r.d0, 'tth': tth})
    return build_problem(group, cell, demand, [sites, *extra_assignments], rows, windows, min_contact, true)


def build_problem(group: SpaceGroup, cell: Dict[str, float], demand: List[dict],
                  label_sets: Sequence[Sequence[Tuple[str, str]]], rows: Sequence[dict],
                  windows: Sequence[dict] = (), min_contact: Optional[float] = None,
                  true_coords: Optional[np.ndarray] = None, overall_b: float = 0.0) -> WyckoffProblem:
    """A search problem from observation rows ({h, k, l, mult, Fo2, sigma, d,
    tth}: |F|^2 per reflection with multiplicity and Lp removed) and one or
    more site assignments ([(element, '4c'), ...] each): the packed reflection
    groups, the scattering table, the assignment and restraint tables and the
    cell's reduced basis."""
    ff_table = load_form_factor_table()
    missing = sorted({d['element'] for d in demand if d['element'] not in ff_table})
    if missing:
        raise ValueError(f'No X-ray scattering factor for {", ".join(missing)}.')
    assignments = [make_assignment(group, demand, a) for a in label_sets]
    tables = build_assignment_tables(assignments, group, demand)
    refl = pack_reflections(rows)
    f_tab, n_elem, _missing = scattering_table(refl, demand, gaussian_form_factor(ff_table), overall_b)
    restraints = build_restraint_tables(demand, list(windows), min_contact)
    red = reduced_cell(cell)
    orth0 = orth_matrix(cell).astype(np.float64)
    true = None
    if true_coords is not None:
        true = np.zeros(tables.max_sites * 3)
        true[:len(true_coords)] = true_coords[:tables.max_sites * 3]
    prob = WyckoffProblem(group, cell, demand, assignments, tables, refl, f_tab, n_elem, restraints,
                          pack_sym_ops(group.ops), has_inversion_at_origin(group.ops), red.orth, red.xform,
                          inverse3(orth0), 1 if restraints.max_distance > red.safe_radius else 0, true, list(rows))
    # penBond / penCoord per charged slot (js/swarm_wyckoff.js:1482-1506)
    n_of = {d['element'].upper(): d['count'] for d in demand}
    bond_slots, coord_centres = 0, 0
    for w in windows:
        nA = n_of.get(str(w['a']).upper(), 0)
        if not nA:
            continue
        has_count = w.get('count') is not None and w['count'] > 0
        if has_count:
            bond_slots += nA * w['count']
            coord_centres += nA
        elif w.get('dmax') is not None:
            bond_slots += nA
            if w.get('bothWays', True) is not False and str(w['a']).upper() != str(w['b']).upper():
                bond_slots += n_of.get(str(w['b']).upper(), 0)
    prob.pen_bond = 0.10 / max(1, bond_slots)
    prob.pen_coord = 0.03 / max(1, coord_centres)
    return prob


# ---------------------------------------------------------------------------
# Batched uneven Wyckoff searches (many independent problems in one launch).
# ---------------------------------------------------------------------------
BATCH_GROUPS = (2, 14, 15, 62, 176, 225)       # P-1, P2_1/c, C2/c, Pnma, P6_3/m, Fm-3m
BATCH_ELEMENTS = ('C', 'N', 'O', 'S', 'Na', 'Cl', 'Ti', 'Fe', 'Pb')


@dataclass
class BatchItem:
    problem: 'WyckoffProblem'
    replicas: int
    points: int
    target_reflections: int


def _log_uniform(rng, lo, hi):
    return float(np.exp(rng.uniform(math.log(lo), math.log(hi))))


def _random_cell(rng, system: str) -> Dict[str, float]:
    a, b, c = (rng.uniform(4.0, 20.0) for _ in range(3))
    if system == 'triclinic':
        return {'a': a, 'b': b, 'c': c, 'alpha': rng.uniform(75, 105), 'beta': rng.uniform(75, 105),
                'gamma': rng.uniform(75, 105)}
    if system == 'monoclinic':
        return {'a': a, 'b': b, 'c': c, 'alpha': 90.0, 'beta': rng.uniform(92, 118), 'gamma': 90.0}
    if system == 'orthorhombic':
        return {'a': a, 'b': b, 'c': c, 'alpha': 90.0, 'beta': 90.0, 'gamma': 90.0}
    if system == 'hexagonal':
        return {'a': a, 'b': a, 'c': c, 'alpha': 90.0, 'beta': 90.0, 'gamma': 120.0}
    return {'a': a, 'b': a, 'c': a, 'alpha': 90.0, 'beta': 90.0, 'gamma': 90.0}


def _cell_volume(cell) -> float:
    al, be, ga = (math.radians(cell[k]) for k in ('alpha', 'beta', 'gamma'))
    return cell['a'] * cell['b'] * cell['c'] * math.sqrt(
        max(1e-12, 1 - math.cos(al) ** 2 - math.cos(be) ** 2 - math.cos(ga) ** 2
            + 2 * math.cos(al) * math.cos(be) * math.cos(ga)))


def batched_problems(n: int = 64, seed: int = 1, max_atoms: int = 512, wavelength: float = 1.5406,
                     max_refl: int = 3000, min_refl: int = 50):
    """Seeded uneven problems: space groups from BATCH_GROUPS, 1-24 sites and
    50-3000 reflections and 2000-12000 points and 256-2048 replicas (all
    log-uniform), cells uniform in 4-20 A, at most ``max_atoms`` atoms per
    cell (resampled otherwise).  The reflection count sets d_min through the
    volume of the reciprocal sphere, kept within [``min_refl``, ``max_refl``]
    by moving d_min (a search whose
    tables do not fit in shared memory next to its eight replica slices reads
    them from global memory); the point count is recorded only (the search's
    fitness works on integrated intensities)."""
    from .symmetry import space_group
    rng = np.random.default_rng(seed)
    out: List[BatchItem] = []
    while len(out) < n:
        g = space_group(int(rng.choice(BATCH_GROUPS)))
        cell = _random_cell(rng, g.system)
        n_sites = max(1, min(24, int(round(_log_uniform(rng, 1, 24)))))
        free = [w for w in g.wyckoff if w.n_free > 0]
        weights = np.array([1.0 / w.multiplicity ** 0.5 for w in free])
        labels, atoms = [], 0
        palette = list(rng.choice(BATCH_ELEMENTS, size=int(rng.integers(1, 5)), replace=False))
        for _ in range(n_sites):
            w = free[int(rng.choice(len(free), p=weights / weights.sum()))]
            el = str(rng.choice(palette))
            labels.append((el, f'{w.multiplicity}{w.letter}'))
            atoms += w.multiplicity
        if atoms > max_atoms:
            continue
        comp: Dict[str, int] = {}
        for el, lab in labels:
            comp[el] = comp.get(el, 0) + int(lab[:-1])
        target = int(round(_log_uniform(rng, 50, 3000)))
        n_pg = len({o.r for o in g.ops})
        n_c = len(g.ops) // n_pg
        vol = _cell_volume(cell)
        dmin = (4 * math.pi * vol / (3 * 2 * n_pg * n_c * target)) ** (1.0 / 3.0)
        dmin = max(dmin, wavelength / 2 * 1.0001)
        pseed = int(rng.integers(1 << 30))
        for _retry in range(8):
            prob = wyckoff_problem(seed=pseed, group_number=g.number, cell=cell,
                                   composition=tuple(comp.items()), sites=tuple(labels), dmin=dmin,
                                   wavelength=wavelength, true_min_contact=1.0, contact_attempts=40)
            if prob.refl.n_refl > max_refl:
                dmin *= 1.02 * (prob.refl.n_refl / max_refl) ** (1.0 / 3.0)
            elif prob.refl.n_refl < min_refl and dmin > wavelength / 2 * 1.0001:
                dmin = max(wavelength / 2 * 1.0001, dmin * 0.98 * (prob.refl.n_refl / min_refl) ** (1.0 / 3.0))
            else:
                break
        if prob.refl.n_refl < min_refl or prob.refl.n_refl > max_refl:
            continue
        replicas = int(round(_log_uniform(rng, 256, 2048) / 8)) * 8
        points = int(round(_log_uniform(rng, 2000, 12000)))
        out.append(BatchItem(prob, replicas, points, target))
    return out


def wyckoff_job(problem: WyckoffProblem, wavelength: float = 1.5406, polarisation_k: float = 1.0,
                **fields) -> dict:
    """A 'wyckoff-search' job message (js/rietveld/rv_solve.js:800-803) for a
    synthetic problem: the group's operators and Wyckoff table, the cell, the
    composition per formula unit with Z, and its reflections as the WPPF
    extraction hands them over (intensity = |F|^2 m Lp, sigma on the same
    scale, 2-theta, d, multiplicity and Lp)."""
    from math import gcd
    g = problem.group
    counts = [d['count'] for d in problem.demand]
    Z = 0
    for c in counts:
        Z = gcd(Z, c)
    formula = ''.join(f"{d['element']}{d['count'] // Z if d['count'] // Z > 1 else ''}" for d in problem.demand)
    hkl = []
    for r in problem.rows:
        th = math.radians(0.5 * r['tth'])
        lp = (1.0 / (math.sin(th) ** 2 * math.cos(th))) * (1 + polarisation_k * math.cos(2 * th) ** 2) / \
            (1 + polarisation_k)
        k = r['mult'] * lp
        hkl.append({'h_orig': r['h'], 'k_orig': r['k'], 'l_orig': r['l'], 'intensity': r['Fo2'] * k,
                    'sigma': r['sigma'] * k, 'multiplicity': r['mult'], 'tth': r['tth'], 'd': r['d'], 'lp': lp})
    job = {'type': 'wyckoff-search', 'cell': dict(problem.cell),
           'symops': [{'xyz': None, 'r': list(o.r), 't_num': list(o.t), 't_den': 24} for o in g.ops],
           'wyckoffTable': [{'letter': w.letter, 'multiplicity': w.multiplicity, 'special_op': w.triplet,
                             'n_free': w.n_free} for w in g.wyckoff],
           'targetComposition': formula, 'wyckoffZ': Z, 'hklList': hkl, 'wavelength': wavelength,
           'polarization': {'K': polarisation_k}, 'applyLP': True, 'seed': 1}
    job.update(fields)
    return job
