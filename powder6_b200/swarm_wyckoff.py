"""Host side of the Wyckoff search on the B200 backend.

Mirrors the device layer of ``runWyckoffSearch`` (js/swarm_wyckoff.js:964-2646):
the same packed buffers, the same per-particle state record, the same
dispatch / evaluate / read / sync operations (``WyckoffSession``), and the
same search schedule -- replica ladders of ``rungs`` chains per assignment
(:1784-1808), exchange every ``swapEvery`` generations (:1825-1851), the
resolution ramp (``rampedGroupCount``, :934-938, :2218-2226) and the penalty
ramp (:2228-2230).  ``run_wyckoff_search`` keeps the whole generation loop on
the device: each CUDA block owns a ladder, so the exchange sweep needs no host
round trip.

``cpu_cross_check`` is the product's FP64 re-score of the winner, the role
``swFitnessOnCpu`` plays in the reference report (js/swarm_wyckoff.js:2524-2563).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import P6WyParticleState, P6WyProblem, check, ptr
from .reflections import ramped_group_count
from .workloads import WyckoffProblem, mulberry32

SW_DEFAULTS = dict(
    penClash=0.05, penBond=0.10, penCoord=0.03, penRampStart=0.2, penRampEnd=4.0, polyProb=0.0,
    tempHot=0.05, tempCold=5e-4, rungs=8, swapEvery=10, stepInit=0.08, stepMin=2e-4, stepMax=0.5,
    targetAccept=0.3, stepAdapt=0.08, rampSteps=24, rampStart=0.25, rampFull=0.6,
    quenchSteps=600, quenchStep0=0.02, quenchStep1=5e-5, topN=20, numParticles=512, generations=2000,
    minParticlesPerAssignment=24,
)

STATE_DTYPE = np.dtype([('fit', '<f4'), ('cc', '<f4'), ('pen', '<f4'), ('step_size', '<f4'), ('temp', '<f4'),
                        ('seed', '<u4'), ('accepted', '<u4'), ('pad', '<u4'), ('best_fit', '<f4'),
                        ('best_cc', '<f4'), ('best_pen', '<f4'), ('best_pad', '<f4')])
assert STATE_DTYPE.itemsize == 48


def adaptation(settings: Optional[dict] = None) -> Dict[str, float]:
    """STEP_UP/STEP_DOWN/STEP_MIN/STEP_MAX as swInject computes and validates them
    (js/swarm_wyckoff.js:201-216)."""
    d = dict(SW_DEFAULTS)
    d.update(settings or {})
    vals = [d['stepMin'], d['stepMax'], d['stepInit'], d['targetAccept'], d['stepAdapt']]
    if (not all(math.isfinite(v) for v in vals) or d['stepMin'] <= 0 or d['stepMax'] < d['stepMin']
            or d['stepInit'] < d['stepMin'] or d['stepInit'] > d['stepMax'] or d['targetAccept'] <= 0
            or d['targetAccept'] >= 1 or d['stepAdapt'] <= 0):
        raise ValueError('Invalid Wyckoff step adaptation settings.')
    out = {'STEP_MIN': d['stepMin'], 'STEP_MAX': d['stepMax'],
           'STEP_UP': math.exp(min(700.0, d['stepAdapt'] * (1 - d['targetAccept']))),
           'STEP_DOWN': math.exp(-d['stepAdapt'] * d['targetAccept'])}
    for k, v in out.items():
        with np.errstate(over='ignore'):
            f = np.float32(v)
        if not np.isfinite(f) or f <= 0:
            raise ValueError('Wyckoff adaptation exceeds GPU float limits.')
    return out


COS_SFU, COS_POLY, COS_FACTORED = 0, 1, 2
COS_NAMES = {COS_SFU: 'sfu', COS_POLY: 'poly', COS_FACTORED: 'factored-fp64'}


def factored_ok(problem: WyckoffProblem) -> bool:
    """The factored FP64 evaluation applies: every rotation of the group is
    diagonal (triclinic, monoclinic and orthorhombic groups)."""
    return all(all(o.r[k] == 0 for k in (1, 2, 3, 5, 6, 7)) for o in problem.group.ops)


def default_cos_mode(problem: WyckoffProblem) -> int:
    """Factored FP64 where the group allows it, else the SFU cosine."""
    return COS_FACTORED if factored_ok(problem) else COS_SFU


class WyckoffSession:
    """One device session: the buffers and kernel of one search (swarm_wyckoff.js:1293-1720).
    ``cos_mode`` None picks ``default_cos_mode``."""

    def __init__(self, problem: WyckoffProblem, num_particles: int, run_key: int = 1,
                 cos_mode: Optional[int] = None, device: int = 0, settings: Optional[dict] = None,
                 max_coord_slots: Optional[int] = None, incremental: int = -1):
        self.lib = _lib.load()
        auto = cos_mode is None
        if auto:
            cos_mode = default_cos_mode(problem) if incremental != 1 else COS_SFU
        self.cos_mode = int(cos_mode)
        self.problem = problem
        self.num_particles = int(num_particles)
        T = problem.tables
        R = problem.restraints
        ad = adaptation(settings)
        self._keep = []

        def arr(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a.ctypes.data_as(C.POINTER(np.ctypeslib.as_ctypes_type(dt)))

        pr = P6WyProblem()
        pr.num_particles = self.num_particles
        pr.gen_pack = arr(T.gen_pack, np.uint32)
        pr.n_assign = len(problem.assignments)
        pr.n_tot = T.n_tot
        pr.sym_packed = arr(problem.sym_packed, np.float32)
        pr.n_ops = len(problem.group.ops)
        pr.site_proj = arr(T.site_proj, np.float32)
        pr.max_sites = T.max_sites
        pr.refl_pack = arr(problem.refl.refl_pack, np.uint32)
        pr.n_refl = problem.refl.n_refl
        pr.group_meta = arr(problem.refl.group_meta, np.float32)
        pr.n_groups = problem.refl.n_groups
        pr.group_stride = problem.refl.group_stride
        pr.f_tab = arr(problem.f_tab, np.float32)
        pr.n_elem = problem.n_elem
        pr.restraint_tables = arr(R.tables, np.float32)
        pr.n_restraint_floats = len(R.tables)
        pr.r_min_off = R.r_min_off
        pr.rule_off = R.rule_off
        pr.n_rules = R.n_rules
        slots = max(64, R.slots_needed) if max_coord_slots is None else max_coord_slots
        pr.max_coord_slots = slots
        pr.geom_slots = slots if R.geometry else 1
        for i in range(9):
            pr.orth[i] = float(problem.orth[i])
            pr.xform[i] = float(problem.xform[i])
            pr.inv_orth[i] = float(problem.inv_orth[i])
        pr.min_image_shell = problem.min_image_shell
        pr.count_shell = 1
        pr.centro = 1 if problem.centro else 0
        pr.pen_clash = problem.pen_clash
        pr.pen_bond = problem.pen_bond
        pr.pen_coord = problem.pen_coord
        pr.pen_geom = problem.pen_geom
        pr.poly_prob = float(min(1.0, max(0.0, (settings or {}).get('polyProb', SW_DEFAULTS['polyProb']))))
        pr.step_up, pr.step_down = ad['STEP_UP'], ad['STEP_DOWN']
        pr.step_min, pr.step_max = ad['STEP_MIN'], ad['STEP_MAX']
        pr.cos_mode = int(cos_mode)
        pr.run_key = int(run_key) & 0xFFFFFFFF
        pr.incremental = int(incremental)
        self.adapt = ad
        h = C.c_void_p()
        st = self.lib.p6_wy_create(C.byref(pr), int(device), C.byref(h))
        if st == _lib.P6_ERR_CAPACITY and auto and cos_mode == COS_FACTORED:
            # the factored tables do not fit next to the replica slices: the SFU cosine reads its tables
            # from global memory instead
            cos_mode = COS_SFU
            self.cos_mode = cos_mode
            pr.cos_mode = cos_mode
            st = self.lib.p6_wy_create(C.byref(pr), int(device), C.byref(h))
        check(st)
        self.h = h
        self.coords_per_particle = T.max_sites * 3

    # -- lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, 'h', None):
            self.lib.p6_wy_destroy(self.h)
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

    # -- reference device operations -------------------------------------------
    def set_assign(self, assign_of: np.ndarray):
        a = np.ascontiguousarray(assign_of, dtype=np.uint32)
        check(self.lib.p6_wy_set_assign(self.h, ptr(a)))

    def set_params(self, n_groups_active: int, pen_scale: float):
        check(self.lib.p6_wy_set_params(self.h, int(n_groups_active), float(pen_scale)))

    def sync_state(self, positions: np.ndarray, state: np.ndarray):
        p = np.ascontiguousarray(positions, dtype=np.float32)
        s = np.ascontiguousarray(state, dtype=STATE_DTYPE)
        check(self.lib.p6_wy_sync_state(self.h, ptr(p), ptr(s)))

    def read_state(self):
        n = self.num_particles * self.coords_per_particle
        pos = np.zeros(n, dtype=np.float32)
        best = np.zeros(n, dtype=np.float32)
        st = np.zeros(self.num_particles, dtype=STATE_DTYPE)
        check(self.lib.p6_wy_read_state(self.h, ptr(pos), ptr(best), ptr(st)))
        return pos, best, st

    def dispatch(self, coords: Optional[np.ndarray] = None, mcmc: bool = False):
        c = None if coords is None else np.ascontiguousarray(coords, dtype=np.float32)
        check(self.lib.p6_wy_dispatch(self.h, ptr(c), 1 if mcmc else 0))

    def evaluate_sync(self, coords: Optional[np.ndarray] = None, mcmc: bool = False):
        c = None if coords is None else np.ascontiguousarray(coords, dtype=np.float32)
        out = np.zeros(2 * self.num_particles, dtype=np.float32)
        check(self.lib.p6_wy_evaluate_sync(self.h, ptr(c), 1 if mcmc else 0, ptr(out)))
        return out[:self.num_particles], out[self.num_particles:]

    # -- fused device path -----------------------------------------------------
    def set_ladders(self, ladders: np.ndarray, rungs: int):
        l = np.ascontiguousarray(ladders, dtype=np.int32)
        check(self.lib.p6_wy_set_ladders(self.h, ptr(l), len(l) // rungs, int(rungs)))

    def set_schedule(self, groups: np.ndarray, pen: np.ndarray):
        g = np.ascontiguousarray(groups, dtype=np.int32)
        p = np.ascontiguousarray(pen, dtype=np.float32)
        check(self.lib.p6_wy_set_schedule(self.h, ptr(g), ptr(p), len(g)))

    def set_quench(self, step_sd: Optional[np.ndarray]):
        """Greedy quench mode (js/swarm_wyckoff.js:2013-2090): per generation step
        width, only improvements accepted, no step adaptation; None restores
        the Metropolis search."""
        if step_sd is None:
            check(self.lib.p6_wy_set_quench(self.h, None, 0))
        else:
            a = np.ascontiguousarray(step_sd, dtype=np.float32)
            check(self.lib.p6_wy_set_quench(self.h, ptr(a), len(a)))

    def run(self, gen0: int, n_gen: int, swap_every: int, reeval_first: bool = True):
        check(self.lib.p6_wy_run(self.h, int(gen0), int(n_gen), int(swap_every), 1 if reeval_first else 0))

    def run_host(self, positions: np.ndarray, state: np.ndarray, gen0: int, n_gen: int, swap_every: int,
                 reeval_first: bool = True):
        n = self.num_particles * self.coords_per_particle
        p = np.ascontiguousarray(positions, dtype=np.float32)
        s = np.ascontiguousarray(state, dtype=STATE_DTYPE)
        pos = np.zeros(n, dtype=np.float32)
        best = np.zeros(n, dtype=np.float32)
        st = np.zeros(self.num_particles, dtype=STATE_DTYPE)
        check(self.lib.p6_wy_run_host(self.h, ptr(p), ptr(s), int(gen0), int(n_gen), int(swap_every),
                                      1 if reeval_first else 0, ptr(pos), ptr(best), ptr(st)))
        return pos, best, st

    def synchronize(self, timeout: float = 60.0):
        check(self.lib.p6_wy_synchronize(self.h, float(timeout)))

    # -- parity support --------------------------------------------------------
    def write_positions_fixed(self, x: np.ndarray):
        a = np.ascontiguousarray(x, dtype=np.uint32)
        check(self.lib.p6_wy_write_positions_fixed(self.h, ptr(a)))

    def set_ladder_split(self, ctas_per_ladder: int):
        """Each ladder of 8 on one 8-warp CTA (1) or a cluster of two 4-warp CTAs (2, default)."""
        check(self.lib.p6_wy_set_ladder_split(self.h, int(ctas_per_ladder)))

    def write_state_fixed(self, current: np.ndarray, best: np.ndarray, state: np.ndarray):
        c = np.ascontiguousarray(current, dtype=np.uint32)
        b = np.ascontiguousarray(best, dtype=np.uint32)
        st = np.ascontiguousarray(state, dtype=STATE_DTYPE)
        check(self.lib.p6_wy_write_state_fixed(self.h, ptr(c), ptr(b), ptr(st)))

    def read_positions_fixed(self):
        n = self.num_particles * self.coords_per_particle
        cur = np.zeros(n, dtype=np.uint32)
        best = np.zeros(n, dtype=np.uint32)
        check(self.lib.p6_wy_read_positions_fixed(self.h, ptr(cur), ptr(best)))
        return cur, best

    def set_trace(self, on: bool):
        check(self.lib.p6_wy_set_trace(self.h, 1 if on else 0))

    def read_trace(self):
        props = np.zeros(self.num_particles * self.coords_per_particle, dtype=np.uint32)
        rec = np.zeros(self.num_particles * 8, dtype=np.float32)
        check(self.lib.p6_wy_read_trace(self.h, ptr(props), ptr(rec)))
        return props, rec.reshape(-1, 8)

    def read_trace_ic(self):
        ic = np.zeros(self.num_particles * self.problem.refl.n_refl, dtype=np.float32)
        check(self.lib.p6_wy_read_trace_ic(self.h, ptr(ic)))
        return ic.reshape(self.num_particles, -1)

    def read_trace_sums(self):
        """FP64 (scc, soo, sco) of each particle's last traced evaluation."""
        out = np.zeros(self.num_particles * 3, dtype=np.float64)
        check(self.lib.p6_wy_read_trace_sums(self.h, ptr(out)))
        return out.reshape(self.num_particles, 3)

    def debug_expand(self, particle: int):
        out = np.zeros(self.problem.n_tot * 3, dtype=np.uint32)
        check(self.lib.p6_wy_debug_expand(self.h, int(particle), ptr(out)))
        return out

    def last_kernel_ms(self) -> float:
        v = C.c_float()
        check(self.lib.p6_wy_last_kernel_ms(self.h, C.byref(v)))
        return v.value

    def query(self) -> dict:
        inc, smem, grid = C.c_int(), C.c_int(), C.c_int()
        check(self.lib.p6_wy_query(self.h, C.byref(inc), C.byref(smem), C.byref(grid)))
        return {'incremental': bool(inc.value), 'smem_bytes': smem.value, 'max_grid': grid.value}

    def launch_count(self) -> int:
        v = C.c_longlong()
        check(self.lib.p6_wy_launch_count(self.h, C.byref(v)))
        return v.value


# ---------------------------------------------------------------------------
# Search schedule
# ---------------------------------------------------------------------------
def build_ladders(assign_of: np.ndarray, rungs: int = 8, temp_cold: float = 5e-4, temp_hot: float = 0.05):
    """Ladders of ``rungs`` chains of one assignment, geometric temperatures from
    cold to hot; leftover chains sit on the cold rung as singleton ladders
    (js/swarm_wyckoff.js:1784-1808).  Returns (ladder table, temperature per chain)."""
    R = max(2, rungs)
    ratio = (temp_hot / temp_cold) ** (1 / (R - 1))
    rung_temp = [temp_cold * ratio ** r for r in range(R)]
    temp = np.zeros(len(assign_of), dtype=np.float32)
    by = {}
    for i, A in enumerate(assign_of):
        by.setdefault(int(A), []).append(i)
    table = []
    for chains in by.values():
        c = 0
        while c + R <= len(chains):
            lad = chains[c:c + R]
            for r, ci in enumerate(lad):
                temp[ci] = rung_temp[r]
            table.extend(lad)
            c += R
        for ci in chains[c:]:
            temp[ci] = rung_temp[0]
            table.extend([ci] + [-1] * (R - 1))
    return np.array(table, dtype=np.int32), temp


def schedule(generations: int, n_groups: int, settings: Optional[dict] = None):
    """nGroupsActive and penScale per generation (js/swarm_wyckoff.js:2218-2230)."""
    d = dict(SW_DEFAULTS)
    d.update(settings or {})
    groups = np.zeros(generations, dtype=np.int32)
    pen = np.zeros(generations, dtype=np.float32)
    for gen in range(generations):
        t = gen / (generations - 1) if generations > 1 else 1.0
        level = min(d['rampSteps'] - 1, int(math.floor(t * d['rampSteps'])))
        groups[gen] = ramped_group_count(n_groups, level, d['rampSteps'] - 1, d['rampStart'], d['rampFull'])
        pen[gen] = d['penRampStart'] + t * (d['penRampEnd'] - d['penRampStart'])
    return groups, pen


def project_all(problem: WyckoffProblem, positions: np.ndarray, assign_of: np.ndarray):
    """projectSites for every particle, vectorised (js/wyckoff_assign.js:1155-1187)."""
    T = problem.tables
    ms = T.max_sites
    P = positions.reshape(len(assign_of), ms, 3).astype(np.float64)
    sp = T.site_proj.reshape(-1, ms, 12).astype(np.float64)[assign_of]        # (n, ms, 12)
    out = np.einsum('nsij,nsj->nsi', sp[:, :, :9].reshape(len(assign_of), ms, 3, 3), P) + sp[:, :, 9:]
    out -= np.floor(out)
    nS = T.site_count[assign_of]
    mask = np.arange(ms)[None, :] < nS[:, None]
    out[~mask] = 0
    return out.reshape(-1).astype(np.float32)


def to_fixed(x: np.ndarray) -> np.ndarray:
    """Fractional coordinates to the kernel's 32-bit fixed point (x mod 1) * 2^32."""
    f = np.asarray(x, dtype=np.float64)
    f = f - np.floor(f)
    v = np.floor(f * 4294967296.0 + 0.5)
    v[v >= 4294967296.0] -= 4294967296.0
    return v.astype(np.uint64).astype(np.uint32)


# ---------------------------------------------------------------------------
# Particle budget over assignments: waves, weighting by dimension, pruning
# (js/wyckoff_assign.js:1188-1278, js/swarm_wyckoff.js:1240-1290, :2291-2337).
# ---------------------------------------------------------------------------
def assignment_dims(problem: WyckoffProblem) -> List[int]:
    """Free parameters of each assignment (at least 1): the particle weights."""
    return [max(1, sum(int(st.w.n_free) for st in A.sites)) for A in problem.assignments]


def weighted_assign(ids: Sequence[int], n: int, min_per: int, weights: Optional[Sequence[float]] = None) -> np.ndarray:
    """Replicas per assignment by largest-remainder (Hamilton) apportionment,
    the allocation rule of js/wyckoff_assign.js:1188-1229: every id gets a
    floor of min(min_per, n // len(ids)); the surplus is shared in proportion
    to the weights (the free-parameter counts), whole parts first, and the
    replicas left over go one each to the largest fractional parts (ties: the
    larger weight, then the earlier id).  The replicas of one assignment are
    contiguous, in the order of ``ids``."""
    out = np.zeros(n, dtype=np.uint32)
    ids = list(ids)
    if not ids:
        return out
    k = len(ids)
    floor_each = min(min_per, n // k)
    w = np.array([max(1e-6, float(weights[a]) if weights is not None and weights[a] else 1.0) for a in ids])
    quota = (n - floor_each * k) * w / w.sum()
    whole = np.floor(quota + 1e-9)
    counts = floor_each + whole.astype(np.int64)
    left = n - int(counts.sum())
    if left > 0:
        order = np.lexsort((np.arange(k), -w, -(quota - whole)))
        counts[order[:left]] += 1
    out[:] = np.repeat(np.array(ids, dtype=np.uint32), counts)
    return out


def prune_assignments(ids: Sequence[int], best: Dict[int, float], keep_fraction: float = 0.5,
                      min_keep: int = 4) -> List[int]:
    """pruneAssignments (js/wyckoff_assign.js:1274-1278): the best
    max(min_keep, ceil(len * keep_fraction)) assignments by best fitness
    (stable for ties; an assignment without a best ranks last)."""
    ranked = sorted(ids, key=lambda a: -best.get(a, -math.inf))
    keep = max(min_keep, math.ceil(len(ranked) * keep_fraction))
    return ranked[:min(keep, len(ranked))]


def assignments_per_wave(n: int, min_per: int = 24, weighted: bool = True) -> int:
    """assignmentsPerWave (js/wyckoff_assign.js:1251-1253)."""
    return max(1, n // (min_per * (2 if weighted else 1)))


def allocate_waves(ids: Sequence[int], n: int, min_per: int = 24,
                   weights: Optional[Sequence[float]] = None) -> List[List[int]]:
    """allocateWaves (js/wyckoff_assign.js:1255-1265): the assignment ids of each wave, in order."""
    per = assignments_per_wave(n, min_per, weights is not None)
    ids = list(ids)
    return [ids[i:i + per] for i in range(0, len(ids), per)]


def initial_state(n: int, temps: np.ndarray, rnd: Callable[[], float], settings: Optional[dict] = None):
    d = dict(SW_DEFAULTS)
    d.update(settings or {})
    st = np.zeros(n, dtype=STATE_DTYPE)
    st['fit'] = -np.inf
    st['cc'] = np.nan
    st['pen'] = 0
    st['step_size'] = d['stepInit']
    st['temp'] = temps
    st['seed'] = [int(rnd() * 4294967296) & 0xFFFFFFFF for _ in range(n)]
    st['best_fit'] = -1e30
    return st


def reflection_intensities(problem: WyckoffProblem, coords: np.ndarray, assign: int = 0) -> np.ndarray:
    """mult |F|^2 of every reflection of one structure in FP64, from the packed
    arrays (the intensities the search kernel forms)."""
    T = problem.tables
    ms = T.max_sites
    sp = T.site_proj[assign * ms * 12:(assign + 1) * ms * 12].astype(np.float64).reshape(ms, 12)
    x = np.asarray(coords, dtype=np.float64).reshape(ms, 3)
    proj = np.einsum('sij,sj->si', sp[:, :9].reshape(ms, 3, 3), x) + sp[:, 9:]
    proj -= np.floor(proj)
    gp = T.gen_pack[assign * T.n_tot:(assign + 1) * T.n_tot].astype(np.int64)
    site, op, ty, skip = gp & 0xFF, (gp >> 8) & 0xFFF, (gp >> 20) & 0xF, (gp >> 24) & 1
    sym = problem.sym_packed.astype(np.float64).reshape(-1, 12)
    R = sym[op, :9].reshape(-1, 3, 3)
    t = sym[op, 9:]
    g = np.einsum('aij,aj->ai', R, proj[site]) + t
    g -= np.floor(g)
    keep = skip == 0
    g, ty = g[keep], np.minimum(ty[keep], problem.n_elem - 1)
    pk = problem.refl.refl_pack[0::2].astype(np.int64)
    hkl = np.stack([(pk & 0x3FF) - 512, ((pk >> 10) & 0x3FF) - 512, ((pk >> 20) & 0x3FF) - 512], 1).astype(np.float64)
    mult = problem.refl.refl_pack[1::2].astype(np.float64)
    q = hkl @ g.T
    ph = 2 * np.pi * (q - np.floor(q))
    f = problem.f_tab.astype(np.float64).reshape(-1, problem.n_elem)[:, ty]
    fr = (f * np.cos(ph)).sum(1)
    fi = (f * np.sin(ph)).sum(1)
    return mult * (fr * fr + fi * fi)


def cpu_cross_check(problem: WyckoffProblem, coords: np.ndarray, assign: int = 0) -> float:
    """FP64 re-score of one structure from the packed arrays (the report's
    cross-check, js/swarm_wyckoff.js:2524-2563)."""
    ic = reflection_intensities(problem, coords, assign)
    gm = problem.refl.group_meta.astype(np.float64).reshape(-1, problem.refl.group_stride)
    scc = soo = sco = 0.0
    for row in gm:
        w = row[3] if problem.refl.group_stride >= 4 else 1.0
        if not w > 0:
            continue
        c = ic[int(row[0]):int(row[0]) + int(row[1])].sum()
        scc += w * c * c
        soo += w * row[2] * row[2]
        sco += w * c * row[2]
    den = scc * soo
    if not den > 1e-20 or not sco > 0:
        return 0.0
    ex = min(1.0, max(0.0, sco * sco / den))
    return min(1.0, max(0.0, 1 - math.sqrt(max(0.0, 1 - ex))))


@dataclass
class SearchResult:
    best_cc: float
    best_pen: float
    best_coords: np.ndarray
    trials: int
    kernel_ms: float
    accept_rate: float
    swap_rate: float
    launches: int
    seed: int
    cpu_check: Dict[str, float] = field(default_factory=dict)
    quench: Dict[str, float] = field(default_factory=dict)
    time_to_target: Optional[float] = None
    wall_s: float = 0.0
    assignments: List[int] = field(default_factory=list)     # the wave's assignments
    kept: List[int] = field(default_factory=list)            # still in contention after the prune
    best_assignment: int = 0
    per_assignment: Dict[int, float] = field(default_factory=dict)   # best cc of each assignment
    bests: Dict[int, dict] = field(default_factory=dict)             # {cc, pen, coords} of each assignment
    screened: Dict[int, float] = field(default_factory=dict)         # screening score (cc - raw pen), if screened
    refined: Dict[int, dict] = field(default_factory=dict)           # {coords, r_start, r, converged} per assignment


def quench_schedule(settings: Optional[dict] = None) -> np.ndarray:
    """Step widths of the quench: geometric from quenchStep0 to quenchStep1 over quenchSteps."""
    d = dict(SW_DEFAULTS)
    d.update(settings or {})
    steps = int(d['quenchSteps'])
    t = np.arange(steps) / max(1, steps - 1) if steps > 1 else np.ones(1)
    return (d['quenchStep0'] * (d['quenchStep1'] / d['quenchStep0']) ** t).astype(np.float32)


def quench(problem: WyckoffProblem, sess: 'WyckoffSession', best: Dict[int, dict], rnd: Callable[[], float],
           settings: Optional[dict] = None) -> Dict[int, dict]:
    """quench (js/swarm_wyckoff.js:2013-2100) on the device: every chain starts
    from its assignment's best, is re-measured at full resolution and the
    final penalty weight, and takes quenchSteps greedy steps of shrinking
    width.  ``best`` maps assignment -> {'cc', 'pen', 'coords'}; returns the
    same map re-scored and improved."""
    d = dict(SW_DEFAULTS)
    d.update(settings or {})
    live = sorted(A for A, b in best.items() if b.get('coords') is not None)
    if not live:
        return best
    n, cpp = sess.num_particles, sess.coords_per_particle
    assign_of = np.array([live[i % len(live)] for i in range(n)], dtype=np.uint32)
    sess.set_assign(assign_of)
    pos = np.concatenate([best[int(A)]['coords'] for A in assign_of]).astype(np.float32)
    st = initial_state(n, np.full(n, d['tempCold'], dtype=np.float32), rnd, d)
    sess.sync_state(pos, st)
    sd = quench_schedule(d)
    steps = len(sd)
    scale = float(d['penRampEnd'])
    sess.set_schedule(np.full(steps, problem.refl.n_groups, dtype=np.int32), np.full(steps, scale, dtype=np.float32))
    sess.set_quench(sd)
    try:
        sess.run(0, steps, 0, True)
        sess.synchronize(600.0)
        ms = sess.last_kernel_ms()
    finally:
        sess.set_quench(None)
    cur, bestpos, st = sess.read_state()
    out = {}
    for A in live:
        idx = np.nonzero(assign_of == A)[0]
        # the start, re-measured at full resolution, is the first candidate
        i0 = int(idx[0])
        rec = [(float(st['best_cc'][i] - st['best_pen'][i] * scale), int(i)) for i in idx if st['best_fit'][i] > -1e29]
        if rec:
            _, i = max(rec)
            out[A] = {'cc': float(st['best_cc'][i]), 'pen': float(st['best_pen'][i]),
                      'coords': bestpos[i * cpp:(i + 1) * cpp].copy(), 'improved': True}
        else:
            out[A] = {'cc': float(st['cc'][i0]), 'pen': float(st['pen'][i0]), 'coords': best[A]['coords'],
                      'improved': False}
    out['_ms'] = ms
    return out


def run_wyckoff_search(problem: WyckoffProblem, num_particles: int = 4096, generations: int = 5000,
                       restarts: int = 1, seed: int = 20261026, cos_mode: Optional[int] = None,
                       chunk: Optional[int] = None,
                       settings: Optional[dict] = None, session: Optional[WyckoffSession] = None,
                       on_progress: Optional[Callable[[dict], None]] = None,
                       should_stop: Optional[Callable[[], bool]] = None, do_quench: bool = True,
                       target_cc: Optional[float] = None, assignment_ids: Optional[Sequence[int]] = None,
                       prune: bool = True, refine: bool = False, world: int = 1) -> SearchResult:
    """One wave of assignments (``assignment_ids``, default all of the
    problem's), ``restarts`` independent restarts, all generations on the
    device, then the quench of the per-assignment bests.  Particles are shared
    out in proportion to each assignment's free parameters (weightedAssign);
    in the first restart, at generation max(20, 0.45 G), a wave of more than
    four assignments keeps the better half (at least four) by best fitness
    and hands the retired assignments' particles to the survivors with fresh
    coordinates and fresh ladders (js/swarm_wyckoff.js:2291-2337).  The
    winner is re-scored at full resolution and the final penalty weight and
    cross-checked on the CPU, as the reference reports.  With ``target_cc``,
    ``time_to_target`` is the wall time from the start to the first chunk
    boundary (or the end of the quench) at which the best cc reached it.
    With ``refine``, the best structure of every assignment is then refined
    by least squares against the grouped |F|^2 (``refine_coordinates``) and
    the result carries the refined coordinates and wR(F^2) in ``refined``.

    Sharded over ``world`` ranks (one process per GPU, each with its own
    replicas, ladders and seed), every rank calls this with the same problem,
    schedule and chunking; at every chunk boundary the per-assignment bests
    are merged over the ranks (``dist.bests_over_ranks``), the prune decides
    on the global bests, a stop request on any rank stops all of them, and
    every rank returns the same per-assignment winners."""
    import time
    from .dist import any_over_ranks, bests_over_ranks, max_per_assignment
    t_start = time.perf_counter()
    d = dict(SW_DEFAULTS)
    d.update(settings or {})
    rnd = mulberry32(seed)
    own = session is None
    sess = session or WyckoffSession(problem, num_particles, run_key=seed, cos_mode=cos_mode, settings=settings)
    n = sess.num_particles
    nA = len(problem.assignments)
    ids = list(range(nA)) if assignment_ids is None else [int(a) for a in assignment_ids]
    if not ids or min(ids) < 0 or max(ids) >= nA:
        raise ValueError('assignment ids out of range')
    wave_ids = list(ids)
    dims = assignment_dims(problem)
    min_per = int(d['minParticlesPerAssignment'])
    assign_of = weighted_assign(ids, n, min_per, dims)
    prune_at = max(20, int(round(generations * 0.45)))
    do_prune = prune and len(ids) > 4 and prune_at < generations
    sess.set_assign(assign_of)
    ladders, temps = build_ladders(assign_of, int(d['rungs']), d['tempCold'], d['tempHot'])
    sess.set_ladders(ladders, max(2, int(d['rungs'])))
    groups, pen = schedule(generations, problem.refl.n_groups, d)
    sess.set_schedule(groups, pen)
    chunk = chunk or generations
    scale = float(pen[-1])
    per_a: Dict[int, dict] = {}
    total_ms = 0.0
    acc_total = 0
    hit = None
    cpp = sess.coords_per_particle

    def record(st, bestpos):
        for i in range(n):
            if not st['best_fit'][i] > -1e29:
                continue
            A = int(assign_of[i])
            f = float(st['best_cc'][i] - st['best_pen'][i] * scale)
            if A not in per_a or f > per_a[A]['cc'] - per_a[A]['pen'] * scale:
                per_a[A] = {'cc': float(st['best_cc'][i]), 'pen': float(st['best_pen'][i]),
                            'coords': bestpos[i * cpp:(i + 1) * cpp].copy()}

    stop = False

    def merge():
        nonlocal per_a
        if world > 1:
            per_a = bests_over_ranks(per_a, nA, cpp, scale, world)

    for restart in range(restarts):
        if stop:
            break
        pos = np.array([rnd() for _ in range(n * cpp)], dtype=np.float32)
        pos = project_all(problem, pos, assign_of)
        st = initial_state(n, temps, rnd, d)
        sess.sync_state(pos, st)
        g0 = 0
        force_eval = False
        while g0 < generations:
            stop = bool(should_stop and should_stop())
            if world > 1:
                stop = any_over_ranks(stop, world)
            if stop:
                break
            end = min(g0 + chunk, generations)
            if restart == 0 and do_prune and g0 < prune_at:
                end = min(end, prune_at)
            ng = end - g0
            reeval = g0 == 0 or groups[g0] != groups[g0 - 1] or force_eval
            force_eval = False
            sess.run(g0, ng, int(d['swapEvery']), reeval)
            sess.synchronize(600.0)
            total_ms += sess.last_kernel_ms()
            g0 += ng
            if world > 1:
                _, bp_sync, st_sync = sess.read_state()
                record(st_sync, bp_sync)
                merge()
            if target_cc is not None and hit is None and g0 < generations:
                if world > 1:
                    reached = any(v['cc'] >= target_cc for v in per_a.values())
                else:
                    _, _, stc = sess.read_state()
                    ok = stc['best_fit'] > -1e29
                    reached = bool(np.any(ok) and float(np.max(stc['best_cc'][ok])) >= target_cc)
                if reached:
                    hit = time.perf_counter() - t_start
            if restart == 0 and do_prune and g0 == prune_at:
                # successive halving on the bests so far, at the current penalty weight
                _, bestpos, stp = sess.read_state()
                record(stp, bestpos)
                now = float(pen[prune_at - 1])
                gbest: Dict[int, float] = {}
                for i in range(n):
                    if stp['best_fit'][i] > -1e29:
                        A = int(assign_of[i])
                        gbest[A] = max(gbest.get(A, -math.inf), float(stp['best_cc'][i] - stp['best_pen'][i] * now))
                gbest = max_per_assignment(gbest, nA, world)
                keep = prune_assignments(ids, gbest, 0.5, 4)
                if len(keep) < len(ids):
                    ids = keep
                    fresh = weighted_assign(ids, n, min_per, dims)
                    moved = fresh != assign_of
                    assign_of = fresh
                    cur_fx, best_fx = sess.read_positions_fixed()
                    rand = np.array([rnd() for _ in range(n * cpp)], dtype=np.float32)
                    newpos = to_fixed(project_all(problem, rand, assign_of)).reshape(n, cpp)
                    cur_fx = cur_fx.reshape(n, cpp)
                    best_fx = best_fx.reshape(n, cpp)
                    cur_fx[moved] = newpos[moved]
                    best_fx[moved] = newpos[moved]
                    stp['fit'][moved] = -np.inf
                    stp['cc'][moved] = np.nan
                    stp['pen'][moved] = 0
                    stp['step_size'][moved] = d['stepInit']
                    stp['best_fit'][moved] = -1e30
                    stp['best_cc'][moved] = 0
                    stp['best_pen'][moved] = 0
                    ladders, temps = build_ladders(assign_of, int(d['rungs']), d['tempCold'], d['tempHot'])
                    stp['temp'] = temps
                    sess.set_assign(assign_of)
                    sess.set_ladders(ladders, max(2, int(d['rungs'])))
                    sess.write_state_fixed(cur_fx.reshape(-1), best_fx.reshape(-1), stp)
                    force_eval = True
            if on_progress:
                info = {'restart': restart + 1, 'restarts': restarts, 'generation': g0,
                        'generations': generations,
                        'fraction': (restart + g0 / generations) / restarts}
                _, bp, sp = sess.read_state()
                ok = np.nonzero(sp['best_fit'] > -1e29)[0]
                if len(ok):
                    now = float(pen[g0 - 1])
                    i = int(ok[np.argmax(sp['best_cc'][ok] - sp['best_pen'][ok] * now)])
                    info.update(best=float(sp['best_cc'][i] - sp['best_pen'][i] * now), cc=float(sp['best_cc'][i]),
                                assignment=int(assign_of[i]), coords=bp[i * cpp:(i + 1) * cpp].copy())
                on_progress(info)
        cur, bestpos, st = sess.read_state()
        acc_total += int(st['accepted'].sum())
        record(st, bestpos)
        merge()
    qinfo = {}
    if do_quench and per_a and not stop:
        before = {A: v['cc'] for A, v in per_a.items()}
        q = quench(problem, sess, per_a, rnd, d)
        qinfo = {'ms': q.pop('_ms'), 'improved': int(sum(1 for A in q if q[A].get('improved'))),
                 'best_before': max(before.values())}
        total_ms += qinfo['ms']
        per_a = q
        merge()
        sess.set_assign(assign_of)
        sess.set_schedule(groups, pen)
    best = {'cc': -np.inf, 'pen': 0.0, 'coords': None, 'A': 0}
    for A, v in per_a.items():
        if v['cc'] - v['pen'] * scale > best['cc'] - best['pen'] * scale:
            best = dict(v, A=A)
    if target_cc is not None and hit is None and best['coords'] is not None and best['cc'] >= target_cc:
        hit = time.perf_counter() - t_start
    if qinfo:
        qinfo['best_after'] = best['cc']
    trials = n * generations * restarts
    res = SearchResult(best['cc'], best['pen'], best['coords'], trials, total_ms,
                       acc_total / max(1, trials), float('nan'), sess.launch_count(), seed, quench=qinfo,
                       time_to_target=hit, wall_s=time.perf_counter() - t_start, assignments=wave_ids,
                       kept=list(ids), best_assignment=int(best['A']),
                       per_assignment={int(A): float(v['cc']) for A, v in per_a.items()},
                       bests={int(A): {'cc': float(v['cc']), 'pen': float(v['pen']), 'coords': v['coords']}
                              for A, v in per_a.items()})
    if best['coords'] is not None:
        cpu = cpu_cross_check(problem, best['coords'], best['A'])
        res.cpu_check = {'gpu': best['cc'], 'cpu': cpu, 'delta': abs(best['cc'] - cpu)}
    if refine and per_a:
        for A in sorted(A for A, v in per_a.items() if v.get('coords') is not None):
            try:
                ref = refine_coordinates(sess, np.asarray(per_a[A]['coords'], dtype=np.float64)[None, :], [A])
            except _lib.P6Error as e:        # e.g. more free coordinates than weighted groups
                res.refined[A] = {'error': str(e)}
                continue
            res.refined[A] = {'coords': ref['coords'][0], 'r_start': float(ref['r_start'][0]),
                              'r': float(ref['r'][0]), 'converged': bool(ref['converged'][0])}
    if own:
        sess.close()
    return res


# The screening stage (WY_LIMITS, js/wyckoff_limits.js:48-53): when the
# assignments need more than FULL_WAVES waves, each is first searched for
# SCREEN_FRACTION of the generations (at least SCREEN_MIN_GENERATIONS, one
# restart), and only the best FULL_WAVES waves' worth get the full search.
FULL_WAVES = 2
SCREEN_FRACTION = 0.1
SCREEN_MIN_GENERATIONS = 60


def rescore_full_resolution(problem: WyckoffProblem, sess: WyckoffSession, bests: Dict[int, dict],
                            seed: int = 1, settings: Optional[dict] = None) -> Dict[int, dict]:
    """rescoreAtFullResolution: each assignment's best structure measured with
    every reflection group and the penalty at weight 1 (one replica per
    assignment, one evaluation launch); returns {A: {cc, pen, coords}}."""
    live = sorted(A for A, b in bests.items() if b.get('coords') is not None)
    if not live:
        return {}
    n = sess.num_particles
    if len(live) > n:
        raise ValueError('more assignments than replicas to re-score them')
    assign_of = np.array([live[i] if i < len(live) else live[0] for i in range(n)], dtype=np.uint32)
    sess.set_assign(assign_of)
    pos = np.concatenate([bests[int(A)]['coords'] for A in assign_of]).astype(np.float32)
    st = initial_state(n, np.full(n, SW_DEFAULTS['tempCold'], dtype=np.float32), mulberry32(seed), settings)
    sess.sync_state(pos, st)
    sess.set_params(problem.refl.n_groups, 1.0)
    sess.dispatch(None, mcmc=False)
    sess.synchronize(60.0)
    _, _, st = sess.read_state()
    return {A: {'cc': float(st['cc'][i]), 'pen': float(st['pen'][i]), 'coords': bests[A]['coords']}
            for i, A in enumerate(live) if np.isfinite(st['cc'][i])}


class P6WyRefineOpts(C.Structure):
    _fields_ = [('max_iter', C.c_int), ('lambda0', C.c_double), ('lambda_up', C.c_double),
                ('lambda_down', C.c_double), ('lambda_max', C.c_double), ('tol_step', C.c_double),
                ('tol_chi', C.c_double), ('max_step', C.c_double)]


REFINE_DEFAULTS = dict(max_iter=60, lambda0=1e-3, lambda_up=10.0, lambda_down=0.4, lambda_max=1e8, tol_step=1e-6,
                       tol_chi=1e-9, max_step=0.05)


def refine_coordinates(sess: WyckoffSession, coords: np.ndarray, assign: Sequence[int],
                       **opts) -> Dict[str, np.ndarray]:
    """refineCoordinatesAgainstWppf (js/coord_refine.js:266-627) on the device for
    a batch of structures: ``coords`` (n x max_sites*3, fractional) against the
    session's grouped |F|^2, each with its assignment.  Returns the refined
    coordinates, the weighted wR(F^2) before and after, chi^2, accepted steps
    and convergence per structure."""
    o = dict(REFINE_DEFAULTS)
    o.update(opts)
    x = np.ascontiguousarray(np.asarray(coords, dtype=np.float64).reshape(len(assign), -1)).copy()
    a = np.ascontiguousarray(assign, dtype=np.uint32)
    n = len(a)
    r0, r1, chi = np.zeros(n), np.zeros(n), np.zeros(n)
    it, cv = np.zeros(n, dtype=np.int32), np.zeros(n, dtype=np.int32)
    ro = P6WyRefineOpts(**o)
    check(sess.lib.p6_wy_refine(sess.h, n, ptr(a), ptr(x), C.cast(C.pointer(ro), C.c_void_p), ptr(r0), ptr(r1),
                                ptr(chi), ptr(it), ptr(cv)))
    return {'coords': x, 'r_start': r0, 'r': r1, 'chi2': chi, 'iterations': it, 'converged': cv.astype(bool)}


def _wave_progress(on_progress: Callable[[dict], None], k: int, waves: int, stage: str):
    """A progress callback that adds the wave and the stage to each report."""
    def report(p: dict):
        q = dict(p, wave=k + 1, waves=waves, stage=stage)
        q['fraction'] = (k + p.get('fraction', 0.0)) / waves
        on_progress(q)
    return report


def run_wyckoff_waves(problem: WyckoffProblem, num_particles: int = 4096, generations: int = 5000,
                      restarts: int = 1, seed: int = 20261026, cos_mode: Optional[int] = None,
                      settings: Optional[dict] = None, session: Optional[WyckoffSession] = None,
                      **kwargs) -> SearchResult:
    """Every assignment of the problem, in waves of assignmentsPerWave in their
    prior order (allocateWaves, js/wyckoff_assign.js:1255-1265;
    js/swarm_wyckoff.js:1262-1290, :2393-2425), each wave one
    ``run_wyckoff_search`` with its own prune.  When they need more than
    FULL_WAVES waves, a screening stage runs first: every assignment for a
    tenth of the generations (at least 60, one restart, no quench), its best
    re-scored at full resolution and penalty weight 1, and only the best
    FULL_WAVES waves' worth, in the order of their scores, get the full
    search.  The result is the best full-search wave's, with the
    per-assignment bests, trials and device time of all waves."""
    d = dict(SW_DEFAULTS)
    d.update(settings or {})
    on_progress = kwargs.pop('on_progress', None)
    should_stop = kwargs.get('should_stop')
    own = session is None
    sess = session or WyckoffSession(problem, num_particles, run_key=seed, cos_mode=cos_mode, settings=settings)
    n, min_per, dims = sess.num_particles, int(d['minParticlesPerAssignment']), assignment_dims(problem)
    all_ids = list(range(len(problem.assignments)))
    screen_results, screened = [], {}
    try:
        kept = all_ids
        if math.ceil(len(all_ids) / assignments_per_wave(n, min_per, True)) > FULL_WAVES:
            g_screen = min(generations, max(SCREEN_MIN_GENERATIONS, int(round(generations * SCREEN_FRACTION))))
            skw = dict(kwargs)
            skw['do_quench'] = False
            skw.pop('target_cc', None)
            bests: Dict[int, dict] = {}
            screen_waves = allocate_waves(all_ids, n, min_per, dims)
            for k, w in enumerate(screen_waves):
                if on_progress is not None:
                    skw['on_progress'] = _wave_progress(on_progress, k, len(screen_waves), 'screen')
                r = run_wyckoff_search(problem, n, g_screen, 1, seed + 104729 * k, cos_mode, settings=settings,
                                       session=sess, assignment_ids=w, **skw)
                screen_results.append(r)
                bests.update(r.bests)
            scored = rescore_full_resolution(problem, sess, bests, seed, settings)
            screened = {A: v['cc'] - v['pen'] for A, v in scored.items()}
            kept = sorted(screened, key=lambda A: -screened[A])[:assignments_per_wave(n, min_per, True) * FULL_WAVES]
            if not kept:
                raise RuntimeError('The screening produced no finite score for any assignment.')
        waves = allocate_waves(kept, n, min_per, dims)
        scale = float(schedule(generations, problem.refl.n_groups, d)[1][-1])
        results = []
        for k, w in enumerate(waves):
            kw = dict(kwargs)
            if on_progress is not None:
                kw['on_progress'] = _wave_progress(on_progress, k, len(waves), 'search')
            results.append(run_wyckoff_search(problem, n, generations, restarts, seed + 7919 * k, cos_mode,
                                              settings=settings, session=sess, assignment_ids=w, **kw))
            if should_stop is not None and should_stop():
                break
    finally:
        if own:
            sess.close()
    best = max(results, key=lambda r: r.best_cc - r.best_pen * scale if r.best_coords is not None else -math.inf)
    out = SearchResult(**{f: getattr(best, f) for f in best.__dataclass_fields__})
    out.trials = sum(r.trials for r in screen_results + results)
    out.kernel_ms = sum(r.kernel_ms for r in screen_results + results)
    out.wall_s = sum(r.wall_s for r in screen_results + results)
    out.assignments = [a for r in results for a in r.assignments]
    out.kept = [a for r in results for a in r.kept]
    out.per_assignment = {A: cc for r in results for A, cc in r.per_assignment.items()}
    out.bests = {A: b for r in results for A, b in r.bests.items()}
    out.screened = screened
    return out
