"""Rigid-fragment Wyckoff search: a molecule with torsions as the searched object.

The reference searches a molecule as independent sites held together by
distance rules (js/molecule_rules.js:1-18 writes a bond and a 1-3 rule per
bond and angle; swarm_reflection.wgsl:893-1130 evaluates them).  Here the
same molecule is searched in direct space: per replica a translation
(fractional), an orientation quaternion and its torsion angles; its atoms are
the sites of the single assignment, in order, so the bond lengths and angles
hold by construction and the structure-factor fitness, clash penalty and
Metropolis acceptance are the search's own (``p6_wy_set_fragment``).

* ``load_molecule``: the config-5 molecule (cimetidine, 17 non-H atoms, from
  the package data derived from the reference's test file).
* ``build_fragment``: reference geometry about its centroid and, for each
  torsion bond, the atoms it turns (the side of the bond away from the
  molecule's first atom).
* ``fragment_coords``: parameters -> fractional coordinates, FP64 (the
  starting coordinates the host writes; the device recomputes them for every
  proposal).
* ``fragment_problem``: the config-5 problem -- P2_1/c, a = 10.2, b = 12.1,
  c = 15.3 A, beta = 100 deg, the molecule on 4e at a random placement and
  conformation, |F|^2 to d_min 1.5 A with 2 % noise.
* ``run_fragment_search``: the device search over fragment parameters
  (ladders, exchange, resolution and penalty ramps, quench from the best).
"""
from __future__ import annotations

import ctypes as C
import json
import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import check, ptr
from .crystal import orth_matrix
from .workloads import DATA, WyckoffProblem, build_problem, load_form_factor_table, mulberry32

N_PARAMS = 16
CIMETIDINE_TORSIONS = ((2, 6), (6, 7), (7, 8), (8, 9), (9, 10), (10, 11))   # the chain between the two groups


class P6WyFragment(C.Structure):
    _fields_ = [('n_atoms', C.c_int), ('n_tors', C.c_int), ('axis_b', C.c_int * 8), ('axis_c', C.c_int * 8),
                ('moving', C.c_uint32 * 8), ('ref_xyz', C.c_double * 96), ('to_frac', C.c_double * 9),
                ('trans_step', C.c_double), ('angle_step', C.c_double)]


@dataclass
class Fragment:
    elements: List[str]
    ref: np.ndarray                      # (n, 3) Cartesian A about the centroid
    torsions: List[Tuple[int, int]]      # (b, c): the turn is about b -> c
    moving: List[int]                    # bit masks of the atoms each torsion turns
    to_frac: np.ndarray                  # (3, 3) Cartesian -> fractional
    trans_step: float = 1.0
    angle_step: float = 2.0 * math.pi
    bonds: List[Tuple[int, int]] = field(default_factory=list)

    @property
    def n_atoms(self) -> int:
        return len(self.elements)

    def as_struct(self) -> P6WyFragment:
        f = P6WyFragment()
        f.n_atoms, f.n_tors = self.n_atoms, len(self.torsions)
        for k, ((b, c), m) in enumerate(zip(self.torsions, self.moving)):
            f.axis_b[k], f.axis_c[k], f.moving[k] = b, c, m
        for i, v in enumerate(self.ref.reshape(-1)):
            f.ref_xyz[i] = float(v)
        for i, v in enumerate(self.to_frac.reshape(-1)):
            f.to_frac[i] = float(v)
        f.trans_step, f.angle_step = self.trans_step, self.angle_step
        return f


def load_molecule(name: str = 'cimetidine') -> Tuple[List[str], np.ndarray, List[Tuple[int, int]]]:
    d = json.loads((DATA / f'{name}_heavy.json').read_text())
    return ([a['element'] for a in d['atoms']], np.array([a['xyz'] for a in d['atoms']], dtype=np.float64),
            [tuple(b) for b in d['bonds']])


def _side(n: int, bonds: Sequence[Tuple[int, int]], b: int, c: int) -> List[int]:
    """Atoms reachable from c without crossing the bond b-c."""
    adj = {i: set() for i in range(n)}
    for u, v in bonds:
        if {u, v} != {b, c}:
            adj[u].add(v)
            adj[v].add(u)
    seen, stack = {c}, [c]
    while stack:
        u = stack.pop()
        for v in adj[u]:
            if v not in seen:
                seen.add(v)
                stack.append(v)
    if b in seen:
        raise ValueError(f'bond {b}-{c} is in a ring: it has no torsion')
    return sorted(seen)


def build_fragment(elements: Sequence[str], xyz: np.ndarray, bonds: Sequence[Tuple[int, int]],
                   torsion_bonds: Sequence[Tuple[int, int]], cell: Dict[str, float]) -> Fragment:
    """The fragment of a molecule: its geometry about the centroid, and per
    torsion bond the atoms on the far side from atom 0 (the turned ones)."""
    xyz = np.asarray(xyz, dtype=np.float64)
    n = len(elements)
    if n > 32 or len(torsion_bonds) > 8:
        raise ValueError('a fragment holds at most 32 atoms and 8 torsions')
    tors, moving = [], []
    for u, v in torsion_bonds:
        side_v = _side(n, bonds, u, v)
        b, c, side = (u, v, side_v) if 0 not in side_v else (v, u, _side(n, bonds, v, u))
        tors.append((b, c))
        moving.append(int(sum(1 << i for i in side)))
    orth = orth_matrix(cell).astype(np.float64).reshape(3, 3)
    return Fragment(list(elements), xyz - xyz.mean(axis=0), tors, moving, np.linalg.inv(orth), bonds=list(bonds))


def _rotate(p: np.ndarray, b: np.ndarray, c: np.ndarray, ang: float) -> np.ndarray:
    u = (c - b) / np.linalg.norm(c - b)
    v = p - b
    return b + v * math.cos(ang) + np.cross(u, v) * math.sin(ang) + np.outer(v @ u, u) * (1 - math.cos(ang))


def quat_matrix(q: Sequence[float]) -> np.ndarray:
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def fragment_coords(frag: Fragment, params: Sequence[float]) -> np.ndarray:
    """Fractional coordinates (n, 3), in [0, 1), of the fragment at ``params``
    (t[3], q[4], torsion angles): the torsions in order, each about its bond as
    the earlier ones left it, then the rotation, the change of basis and the
    translation."""
    p = np.asarray(params, dtype=np.float64)
    x = frag.ref.copy()
    for k, ((b, c), m) in enumerate(zip(frag.torsions, frag.moving)):
        idx = [i for i in range(frag.n_atoms) if (m >> i) & 1]
        x[idx] = _rotate(x[idx], x[b].copy(), x[c].copy(), float(p[7 + k]))
    cart = x @ quat_matrix(p[3:7]).T
    f = cart @ frag.to_frac.T + p[:3]
    return f - np.floor(f)


def random_params(rng: np.random.Generator, n: int, n_tors: int) -> np.ndarray:
    """n uniformly random placements: translation in the cell, orientation
    uniform on the rotation group, torsions uniform in [-pi, pi)."""
    out = np.zeros((n, N_PARAMS), dtype=np.float64)
    out[:, :3] = rng.random((n, 3))
    q = rng.normal(size=(n, 4))
    out[:, 3:7] = q / np.linalg.norm(q, axis=1, keepdims=True)
    out[:, 7:7 + n_tors] = rng.uniform(-math.pi, math.pi, size=(n, n_tors))
    return out


def fragment_problem(seed: int = 1, dmin: float = 1.5, noise: float = 0.02, min_contact: float = 1.0,
                     wavelength: float = 1.5406) -> Tuple[WyckoffProblem, Fragment, np.ndarray]:
    """Config 5 in direct space: cimetidine (C10N6S, 17 non-H atoms) on 4e of
    P2_1/c, a = 10.2, b = 12.1, c = 15.3 A, beta = 100 deg, at a seeded random
    placement and conformation whose shortest intermolecular contact is at
    least 2.5 A; |F|^2 of every unique reflection to d_min with X-ray f(s) and
    2 % Gaussian noise.  Returns the problem (17 sites, one assignment), the
    fragment and the true parameters."""
    from .reflections import gaussian_form_factor, generate_reflections
    from .symmetry import space_group
    from .workloads import structure_factors_fp64
    cell = {'a': 10.2, 'b': 12.1, 'c': 15.3, 'alpha': 90.0, 'beta': 100.0, 'gamma': 90.0}
    group = space_group(14)
    elements, xyz, bonds = load_molecule()
    frag = build_fragment(elements, xyz, bonds, CIMETIDINE_TORSIONS, cell)
    ff_table = load_form_factor_table()
    order = []
    for e in elements:
        if e not in order:
            order.append(e)
    demand = [{'element': e, 'count': 4 * elements.count(e), 'z': ff_table[e]['Z']} for e in order]
    labels = [(e, '4e') for e in elements]
    rng = np.random.default_rng(seed)
    orth = orth_matrix(cell).astype(np.float64).reshape(3, 3)
    for _ in range(500):
        truth = random_params(rng, 1, len(frag.torsions))[0]
        f = fragment_coords(frag, truth)
        if _clear(group, f, orth, frag, 2.5):
            break
    from .wyckoff_tables import make_assignment
    assignment = make_assignment(group, demand, labels)
    refs = generate_reflections(cell, group.ops, dmin, with_eq=False)
    hkl = np.array([[r.h, r.k, r.l] for r in refs], dtype=np.int64)
    ff = gaussian_form_factor(ff_table)
    f_of = np.array([[ff(d['element'], 1.0 / r.d0) for d in demand] for r in refs])
    I = structure_factors_fp64(group, assignment, f.reshape(-1), hkl, f_of)
    floor_ = 1e-3 * float(np.mean(I))
    rows = []
    for r, i_true in zip(refs, I):
        sigma = noise * max(i_true, floor_)
        tth = 2 * math.degrees(math.asin(min(1.0, wavelength / (2 * r.d0))))
        rows.append({'h': r.h, 'k': r.k, 'l': r.l, 'mult': r.m, 'Fo2': i_true + rng.normal() * sigma,
                     'sigma': sigma, 'd': r.d0, 'tth': tth})
    prob = build_problem(group, cell, demand, [labels], rows, (), min_contact, f.reshape(-1))
    return prob, frag, truth


def _clear(group, f: np.ndarray, orth: np.ndarray, frag: Fragment, dmin: float) -> bool:
    """Every atom of the molecule is at least dmin from every atom of its
    symmetry and lattice copies (the molecule itself excluded)."""
    shifts = np.array([[i, j, k] for i in (-1, 0, 1) for j in (-1, 0, 1) for k in (-1, 0, 1)], dtype=np.float64)
    for oi, o in enumerate(group.ops):
        R = np.array(o.r, dtype=np.float64).reshape(3, 3)
        img = f @ R.T + np.array(o.t_frac)
        img -= np.floor(img)
        for sft in shifts:
            if oi == 0 and not np.any(sft):
                continue
            d = f[:, None, :] - (img + sft)[None, :, :]
            if np.min(np.linalg.norm(d @ orth.T, axis=-1)) < dmin:
                return False
    return True


def set_fragment(sess, frag: Optional[Fragment]):
    if frag is None:
        check(sess.lib.p6_wy_set_fragment(sess.h, None))
        return
    f = frag.as_struct()
    check(sess.lib.p6_wy_set_fragment(sess.h, C.cast(C.pointer(f), C.c_void_p)))


def write_fragment_state(sess, params: np.ndarray):
    a = np.ascontiguousarray(np.asarray(params, dtype=np.float32).reshape(sess.num_particles, N_PARAMS))
    check(sess.lib.p6_wy_write_fragment_state(sess.h, ptr(a)))


def read_fragment_state(sess) -> Tuple[np.ndarray, np.ndarray]:
    cur = np.zeros((sess.num_particles, N_PARAMS), dtype=np.float32)
    best = np.zeros_like(cur)
    check(sess.lib.p6_wy_read_fragment_state(sess.h, ptr(cur), ptr(best)))
    return cur, best


def device_coords(sess, frag: Fragment, params: np.ndarray) -> np.ndarray:
    """The device's fixed-point mapping of parameter vectors: (n, atoms, 3) words."""
    p = np.ascontiguousarray(np.asarray(params, dtype=np.float32).reshape(-1, N_PARAMS))
    out = np.zeros(len(p) * frag.n_atoms * 3, dtype=np.uint32)
    check(sess.lib.p6_wy_debug_fragment(sess.h, ptr(p), len(p), ptr(out)))
    return out.reshape(len(p), frag.n_atoms, 3)


@dataclass
class FragmentResult:
    best_cc: float
    best_pen: float
    best_params: np.ndarray
    best_coords: np.ndarray
    trials: int
    kernel_ms: float
    time_to_target: Optional[float] = None
    trace: List[Tuple[float, float]] = field(default_factory=list)   # (seconds, best cc) at each chunk


def run_fragment_search(problem: WyckoffProblem, frag: Fragment, num_particles: int = 8192, generations: int = 2000,
                        seed: int = 1, chunk: int = 100, target_cc: Optional[float] = None,
                        session=None, do_quench: bool = True, settings: Optional[dict] = None,
                        start: Optional[np.ndarray] = None, full_resolution: bool = False) -> FragmentResult:
    """The search over fragment parameters on the device: replica ladders of 8
    with exchange every 10 generations, the reference's resolution and
    penalty ramps (or every group at the final penalty weight throughout,
    ``full_resolution``), generations in chunks (the best read between
    launches for the time to target), then the quench of the best structure.
    ``start``: the replicas' starting parameters (n x 16); random placements
    otherwise."""
    from .swarm_wyckoff import (SW_DEFAULTS, WyckoffSession, build_ladders, initial_state, quench_schedule,
                                schedule)
    t0 = time.perf_counter()
    d = dict(SW_DEFAULTS)
    d.update(settings or {})
    own = session is None
    sess = session or WyckoffSession(problem, num_particles, run_key=seed, settings=settings)
    n, cpp = sess.num_particles, sess.coords_per_particle
    set_fragment(sess, frag)
    assign = np.zeros(n, dtype=np.uint32)
    sess.set_assign(assign)
    ladders, temps = build_ladders(assign, int(d['rungs']), d['tempCold'], d['tempHot'])
    sess.set_ladders(ladders, int(d['rungs']))
    groups, pen = schedule(generations, problem.refl.n_groups, d)
    if full_resolution:
        groups[:] = problem.refl.n_groups
        pen[:] = pen[-1]
    sess.set_schedule(groups, pen)
    rng = np.random.default_rng(seed)
    prm = random_params(rng, n, len(frag.torsions)) if start is None else np.asarray(start, dtype=np.float64)
    pos = np.zeros((n, cpp), dtype=np.float32)
    for i in range(n):
        pos[i, :frag.n_atoms * 3] = fragment_coords(frag, prm[i]).reshape(-1)
    st = initial_state(n, temps, mulberry32(seed), d)
    sess.sync_state(pos.reshape(-1), st)
    write_fragment_state(sess, prm)
    res = FragmentResult(-np.inf, 0.0, None, None, n * generations, 0.0)
    scale = float(pen[-1])
    g0 = 0
    while g0 < generations:
        ng = min(chunk, generations - g0)
        sess.run(g0, ng, int(d['swapEvery']), g0 == 0 or groups[g0] != groups[g0 - 1])
        sess.synchronize(600.0)
        res.kernel_ms += sess.last_kernel_ms()
        g0 += ng
        _, _, stc = sess.read_state()
        ok = stc['best_fit'] > -1e29
        b = float(np.max(stc['best_cc'][ok])) if np.any(ok) else float('nan')
        res.trace.append((time.perf_counter() - t0, b))
        if target_cc is not None and res.time_to_target is None and b >= target_cc:
            res.time_to_target = time.perf_counter() - t0
    _, bestpos, st = sess.read_state()
    _, bprm = read_fragment_state(sess)
    ok = np.nonzero(st['best_fit'] > -1e29)[0]
    i = int(ok[np.argmax(st['best_cc'][ok] - st['best_pen'][ok] * scale)])
    best_prm, best_pos = bprm[i].copy(), bestpos[i * cpp:(i + 1) * cpp].copy()
    res.best_cc, res.best_pen = float(st['best_cc'][i]), float(st['best_pen'][i])
    if do_quench:
        # every chain from the best structure, greedy steps of shrinking width at full resolution
        sd = quench_schedule(d)
        sess.sync_state(np.tile(best_pos, n), initial_state(n, np.full(n, d['tempCold'], dtype=np.float32),
                                                             mulberry32(seed + 1), d))
        write_fragment_state(sess, np.tile(best_prm, (n, 1)))
        sess.set_schedule(np.full(len(sd), problem.refl.n_groups, dtype=np.int32),
                          np.full(len(sd), scale, dtype=np.float32))
        sess.set_quench(sd)
        try:
            sess.run(0, len(sd), 0, True)
            sess.synchronize(600.0)
            res.kernel_ms += sess.last_kernel_ms()
        finally:
            sess.set_quench(None)
            sess.set_schedule(groups, pen)
        _, bestpos, st = sess.read_state()
        _, bprm = read_fragment_state(sess)
        ok = np.nonzero(st['best_fit'] > -1e29)[0]
        j = int(ok[np.argmax(st['best_cc'][ok] - st['best_pen'][ok] * scale)])
        if st['best_cc'][j] - st['best_pen'][j] * scale >= res.best_cc - res.best_pen * scale:
            res.best_cc, res.best_pen = float(st['best_cc'][j]), float(st['best_pen'][j])
            best_prm, best_pos = bprm[j].copy(), bestpos[j * cpp:(j + 1) * cpp].copy()
        if target_cc is not None and res.time_to_target is None and res.best_cc >= target_cc:
            res.time_to_target = time.perf_counter() - t0
    res.best_params, res.best_coords = best_prm, best_pos
    if own:
        sess.close()
    return res


def run_fragment_pattern_search(problem: WyckoffProblem, frag: Fragment, pp, method: int, num_particles: int = 8192,
                                generations: int = 15000, seed: int = 1, chunk: int = 500,
                                target_rwp: Optional[float] = None, settings: Optional[dict] = None) -> dict:
    """The rigid-fragment search scored on a powder pattern (``pp``, a
    ProfileProblem of ``problem``): every reflection at the final penalty
    weight from random placements, with the pattern's chi^2 at the best scale
    from the split-BF16 or FP32 contraction (``p6_wy_profile_run``) or in
    Gram form inside the fused search (``GRAM_FP64``).  The clock runs from
    the first evaluation (the host's drawing and upload of the start
    excluded) to the first chunk boundary at or below ``target_rwp``.
    Returns best_rwp, time_to_target, generations_to_target, device_ms."""
    from .contraction import ContractionSession
    from .profile_search import GRAM_FP64, METHOD_NAMES, PatternGram, _ContractionInput, gram_operands, \
        set_session_pattern
    from .swarm_wyckoff import SW_DEFAULTS, WyckoffSession, build_ladders, initial_state, schedule
    d = dict(SW_DEFAULTS)
    d.update(settings or {})
    swap = int(d['swapEvery'])
    with WyckoffSession(problem, num_particles, run_key=seed, settings=settings) as sess:
        n, cpp = sess.num_particles, sess.coords_per_particle
        set_fragment(sess, frag)
        assign = np.zeros(n, dtype=np.uint32)
        sess.set_assign(assign)
        ladders, temps = build_ladders(assign, int(d['rungs']), d['tempCold'], d['tempHot'])
        sess.set_ladders(ladders, int(d['rungs']))
        groups, pen = schedule(generations, problem.refl.n_groups, d)
        groups[:] = problem.refl.n_groups
        pen[:] = pen[-1]
        sess.set_schedule(groups, pen)
        rng = np.random.default_rng(seed)
        prm = random_params(rng, n, len(frag.torsions))
        pos = np.zeros((n, cpp), dtype=np.float32)
        for i in range(n):
            pos[i, :frag.n_atoms * 3] = fragment_coords(frag, prm[i]).reshape(-1)
        sess.sync_state(pos.reshape(-1), initial_state(n, temps, mulberry32(seed), d))
        write_fragment_state(sess, prm)
        ct = None
        if method == GRAM_FP64:
            v, band, bw, syy = gram_operands(pp)
            set_session_pattern(sess, PatternGram(v, band, bw, syy, pp.n_points, pp.rwp_true))
            sess.set_params(problem.refl.n_groups, float(pen[-1]))
        else:
            ct = ContractionSession(_ContractionInput(pp), max_replicas=n)
            ct.set_fitted(True)
        try:
            sess.synchronize(600.0)
            t0 = time.perf_counter()
            if ct is None:
                sess.dispatch(None, mcmc=False)
            else:
                check(sess.lib.p6_wy_profile_run(sess.h, ct.h, int(method), 0, 0, swap, 1, 0))
            sess.synchronize(600.0)
            dev_ms = sess.last_kernel_ms()
            hit, hit_gen, g0 = None, None, 0
            while g0 < generations:
                ng = min(chunk, generations - g0)
                if ct is None:
                    sess.run(g0, ng, swap, False)
                else:
                    check(sess.lib.p6_wy_profile_run(sess.h, ct.h, int(method), g0, ng, swap, 0, 0))
                sess.synchronize(600.0)
                dev_ms += sess.last_kernel_ms()
                g0 += ng
                if target_rwp is not None and hit is None:
                    _, _, st = sess.read_state()
                    ok = st['best_fit'] > -1e29
                    if np.any(ok) and 1.0 - float(np.max(st['best_cc'][ok])) <= target_rwp:
                        hit, hit_gen = time.perf_counter() - t0, g0
                        break
            _, _, st = sess.read_state()
            ok = st['best_fit'] > -1e29
            best = 1.0 - float(np.max(st['best_cc'][ok])) if np.any(ok) else 1.0
            return {'method': METHOD_NAMES[method], 'seed': seed, 'best_rwp': best, 'time_to_target': hit,
                    'generations_to_target': hit_gen, 'generations': g0, 'device_ms': dev_ms}
        finally:
            if ct is not None:
                ct.close()


def main(argv=None):
    """python -m powder6_b200.fragment: a short search of config 5's rigid
    fragment against its pattern with each method named; one JSON line per
    method."""
    import argparse
    from .profile_search import METHOD_NAMES, profile_problem
    names = {v: k for k, v in METHOD_NAMES.items()}
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument('--replicas', type=int, default=8192)
    ap.add_argument('--generations', type=int, default=100)
    ap.add_argument('--methods', default='split3-bf16,fp32-dense,gram-fp64', help=', '.join(names))
    ap.add_argument('--seed', type=int, default=11)
    a = ap.parse_args(argv)
    P, frag, _ = fragment_problem(seed=1)
    pp = profile_problem(P, seed=1)
    for m in a.methods.split(','):
        r = run_fragment_pattern_search(P, frag, pp, names[m], a.replicas, a.generations, seed=a.seed,
                                        chunk=a.generations)
        r['us_per_generation'] = 1000.0 * r['device_ms'] / max(1, r['generations'])
        print(json.dumps(r), flush=True)


if __name__ == '__main__':
    main()
