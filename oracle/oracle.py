"""ORACLE -- test infrastructure, not product code.

ctypes access to libp6oracle.so, the FP64 CPU restatement of the reference's
trial evaluation (see p6_oracle_wyckoff.c for the functions and the reference
lines each follows).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg import this module; the product path never does.
"""
from __future__ import annotations

import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / 'libp6oracle.so'


class Geom(C.Structure):
    _fields_ = [('o', C.c_double * 9), ('r', C.c_double * 9), ('minImageShell', C.c_int), ('countShell', C.c_int),
                ('penClash', C.c_double), ('penBond', C.c_double), ('penCoord', C.c_double),
                ('penGeom', C.c_double), ('penScale', C.c_double)]


class Problem(C.Structure):
    _fields_ = [('genPack', C.c_void_p), ('symPacked', C.c_void_p), ('siteProj', C.c_void_p),
                ('reflPack', C.c_void_p), ('groupMeta', C.c_void_p), ('fTab', C.c_void_p), ('tables', C.c_void_p),
                ('nTot', C.c_int), ('maxSites', C.c_int), ('nElem', C.c_int), ('nGroupsActive', C.c_int),
                ('stride', C.c_int), ('rMinOff', C.c_int), ('ruleOff', C.c_int), ('nRules', C.c_int),
                ('maxCoordSlots', C.c_int), ('geomSlots', C.c_int), ('centro', C.c_int),
                ('stepUp', C.c_double), ('stepDown', C.c_double), ('stepMin', C.c_double), ('stepMax', C.c_double)]


_lib = None


def build():
    if not LIB.exists() or any(p.stat().st_mtime > LIB.stat().st_mtime for p in HERE.glob('*.c')):
        subprocess.run(['make', '-s', '-C', str(HERE)], check=True)


def load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(str(LIB))
        P = C.c_void_p
        lib.p6o_wy_fitness.restype = C.c_double
        lib.p6o_wy_fitness.argtypes = [P, C.c_int, P, P, C.c_int, P, P, C.c_int, C.c_int, P, P, C.c_int, C.c_int, P]
        lib.p6o_wy_fitness_projected.restype = C.c_double
        lib.p6o_wy_fitness_projected.argtypes = [P, P, C.c_int, P, P, C.c_int, C.c_int, P, P, C.c_int, C.c_int, P]
        lib.p6o_wy_expand_fixed.restype = None
        lib.p6o_wy_expand_fixed.argtypes = [P, P, C.c_int, P, P, P]
        lib.p6o_wy_penalty_sites.restype = C.c_double
        lib.p6o_wy_penalty_sites.argtypes = [P, P, C.c_int, P, C.c_int, P, C.c_int, C.c_int, C.c_int, C.c_int,
                                             C.c_int, C.POINTER(Geom)]
        lib.p6o_wy_accept.restype = C.c_int
        lib.p6o_wy_accept.argtypes = [P, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_double, C.POINTER(C.c_int)]
        lib.p6o_wy_generation.restype = C.c_long
        lib.p6o_wy_generation.argtypes = [C.POINTER(Problem), C.POINTER(Geom), C.c_int, P, P, P, P, C.c_int]
        lib.p6o_num_threads.restype = C.c_int
        lib.p6o_num_threads.argtypes = []
        if hasattr(lib, 'p6o_philox'):
            lib.p6o_philox.restype = None
            lib.p6o_philox.argtypes = [P, P, P]
        _lib = lib
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data)


def wy_fitness(coords, site_proj_row, gen_pack_row, sym_packed, group_meta, n_groups, stride, refl_pack, f_tab,
               n_elem, centro):
    """swFitnessOnCpu: returns (cc, (scc, soo, sco))."""
    lib = load()
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    sp = np.ascontiguousarray(site_proj_row, dtype=np.float32)
    gp = np.ascontiguousarray(gen_pack_row, dtype=np.uint32)
    sums = np.zeros(3)
    cc = lib.p6o_wy_fitness(_p(coords), len(coords) // 3, _p(sp), _p(gp), len(gp), _p(sym_packed),
                            _p(group_meta), n_groups, stride, _p(refl_pack), _p(f_tab), n_elem, int(centro),
                            _p(sums))
    return cc, tuple(sums)


def wy_fitness_projected(proj, gen_pack_row, sym_packed, group_meta, n_groups, stride, refl_pack, f_tab, n_elem,
                         centro):
    lib = load()
    proj = np.ascontiguousarray(proj, dtype=np.float64)
    gp = np.ascontiguousarray(gen_pack_row, dtype=np.uint32)
    sums = np.zeros(3)
    cc = lib.p6o_wy_fitness_projected(_p(proj), _p(gp), len(gp), _p(sym_packed), _p(group_meta), n_groups, stride,
                                      _p(refl_pack), _p(f_tab), n_elem, int(centro), _p(sums))
    return cc, tuple(sums)


def expand_fixed(site_x, gen_pack_row, rint, tfix):
    lib = load()
    site_x = np.ascontiguousarray(site_x, dtype=np.uint32)
    gp = np.ascontiguousarray(gen_pack_row, dtype=np.uint32)
    rint = np.ascontiguousarray(rint, dtype=np.int32)
    tfix = np.ascontiguousarray(tfix, dtype=np.uint32)
    out = np.zeros(len(gp) * 3, dtype=np.uint32)
    lib.p6o_wy_expand_fixed(_p(site_x), _p(gp), len(gp), _p(rint), _p(tfix), _p(out))
    return out


def make_geom(orth, xform, min_image_shell, count_shell, pen_clash, pen_bond, pen_coord, pen_geom, pen_scale):
    g = Geom()
    for i in range(9):
        g.o[i] = float(orth[i])
        g.r[i] = float(xform[i])
    g.minImageShell = int(min_image_shell)
    g.countShell = int(count_shell)
    g.penClash, g.penBond, g.penCoord, g.penGeom, g.penScale = (float(pen_clash), float(pen_bond),
                                                                  float(pen_coord), float(pen_geom), float(pen_scale))
    return g


def wy_penalty(proj, gen_pack_row, sym_packed, n_elem, tables, r_min_off, rule_off, n_rules, max_coord_slots,
               geom_slots, geom):
    lib = load()
    proj = np.ascontiguousarray(proj, dtype=np.float64)
    gp = np.ascontiguousarray(gen_pack_row, dtype=np.uint32)
    tables = np.ascontiguousarray(tables, dtype=np.float32)
    return lib.p6o_wy_penalty_sites(_p(proj), _p(gp), len(gp), _p(sym_packed), n_elem, _p(tables), r_min_off,
                                    rule_off, n_rules, max_coord_slots, geom_slots, C.byref(geom))


def wy_accept(state8, cc, pen, pen_scale, u, step_up, step_down, step_min, step_max):
    lib = load()
    st = np.ascontiguousarray(state8, dtype=np.float64).copy()
    bu = C.c_int(0)
    acc = lib.p6o_wy_accept(_p(st), cc, pen, pen_scale, u, step_up, step_down, step_min, step_max, C.byref(bu))
    return acc, st, bu.value


def num_threads():
    return load().p6o_num_threads()


class WyckoffCpuRunner:
    """Whole generations of the Wyckoff search on the host cores (FP64, OpenMP
    over replicas): the timed CPU baseline.  Holds the packed arrays alive."""

    def __init__(self, P, n_particles, seed=1, n_threads=0, step_up=None, step_down=None):
        import math as _m
        self.lib = load()
        self.P = P
        self.n = int(n_particles)
        self.keep = []

        def k(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            self.keep.append(a)
            return a.ctypes.data

        pr = Problem()
        pr.genPack = k(P.tables.gen_pack, np.uint32)
        pr.symPacked = k(P.sym_packed, np.float32)
        pr.siteProj = k(P.tables.site_proj, np.float32)
        pr.reflPack = k(P.refl.refl_pack, np.uint32)
        pr.groupMeta = k(P.refl.group_meta, np.float32)
        pr.fTab = k(P.f_tab, np.float32)
        pr.tables = k(P.restraints.tables, np.float32)
        pr.nTot, pr.maxSites, pr.nElem = P.n_tot, P.max_sites, P.n_elem
        pr.nGroupsActive, pr.stride = P.refl.n_groups, P.refl.group_stride
        pr.rMinOff, pr.ruleOff, pr.nRules = P.restraints.r_min_off, P.restraints.rule_off, P.restraints.n_rules
        pr.maxCoordSlots = max(64, P.restraints.slots_needed)
        pr.geomSlots = pr.maxCoordSlots if P.restraints.geometry else 1
        pr.centro = 1 if P.centro else 0
        pr.stepUp = step_up if step_up is not None else _m.exp(0.08 * 0.7)
        pr.stepDown = step_down if step_down is not None else _m.exp(-0.08 * 0.3)
        pr.stepMin, pr.stepMax = 2e-4, 0.5
        self.pr = pr
        rng = np.random.default_rng(seed)
        ms = P.max_sites
        sp = P.tables.site_proj[:ms * 12].astype(np.float64).reshape(ms, 12)
        raw = rng.random((self.n, ms, 3))
        pos = np.einsum('sij,nsj->nsi', sp[:, :9].reshape(ms, 3, 3), raw) + sp[:, 9:]
        self.pos = np.ascontiguousarray((pos - np.floor(pos)).reshape(-1))
        self.assign = np.zeros(self.n, dtype=np.uint32)
        R = 8
        ratio = (0.05 / 5e-4) ** (1 / (R - 1))
        st = np.zeros((self.n, 8))
        st[:, 0] = -1e30
        st[:, 3] = 0.08
        st[:, 4] = [5e-4 * ratio ** (i % R) for i in range(self.n)]
        st[:, 5] = -1e30
        self.st = np.ascontiguousarray(st.reshape(-1))
        self.seeds = rng.integers(1, 2 ** 32 - 1, size=self.n, dtype=np.uint64).astype(np.uint32)
        self.n_threads = int(n_threads)

    def generation(self, n_groups_active, pen_scale):
        self.pr.nGroupsActive = int(n_groups_active)
        P = self.P
        g = make_geom(P.orth, P.xform, P.min_image_shell, 1, P.pen_clash, P.pen_bond, P.pen_coord, P.pen_geom,
                      pen_scale)
        return self.lib.p6o_wy_generation(C.byref(self.pr), C.byref(g), self.n, _p(self.pos), _p(self.assign),
                                          _p(self.st), _p(self.seeds), self.n_threads)


# ---------------------------------------------------------------------------
# Parallel-tempering Rietveld cost (p6_oracle_pt.c)
# ---------------------------------------------------------------------------
class PtProblem(C.Structure):
    _fields_ = [('nOps', C.c_int), ('rot', C.c_void_p), ('trans', C.c_void_p),
                ('nReps', C.c_int), ('repRot', C.c_void_p), ('repTrans', C.c_void_p),
                ('nAtoms', C.c_int), ('pos', C.c_void_p), ('wMult', C.c_void_p), ('occ', C.c_void_p),
                ('ffA', C.c_void_p), ('ffB', C.c_void_p), ('ffC', C.c_void_p),
                ('n', C.c_int), ('tth', C.c_void_p), ('y', C.c_void_p), ('w', C.c_void_p),
                ('lambda1', C.c_double), ('lambda2', C.c_double), ('ratio', C.c_double), ('polK', C.c_double),
                ('minFwhm', C.c_double), ('nBkg', C.c_int), ('dmin', C.c_double),
                ('hasPo', C.c_int), ('poDir', C.c_double * 3), ('hasAsym', C.c_int), ('method', C.c_int),
                ('hasShift', C.c_int)]


class PtSetup(C.Structure):
    _fields_ = [('nv', C.c_int), ('index', C.c_void_p), ('lo', C.c_void_p), ('hi', C.c_void_p),
                ('scales', C.c_void_p), ('cubic', C.c_int), ('chains', C.c_int), ('sweeps', C.c_int),
                ('maxTemp', C.c_double), ('seed', C.c_uint32)]


class PtModel:
    """FP64 reference cost of a powder6_b200.pt_gpu.PTProblem (the same inputs the kernel gets)."""

    def __init__(self, prob, dmin=None):
        from powder6_b200.symmetry import cosets, space_group
        lib = load()
        lib.p6o_pt_cost.restype = C.c_double
        lib.p6o_pt_cost.argtypes = [C.POINTER(PtProblem), C.c_void_p, C.c_void_p, C.c_void_p]
        lib.p6o_pt_temper.restype = C.c_double
        lib.p6o_pt_temper.argtypes = [C.POINTER(PtProblem), C.POINTER(PtSetup), C.c_void_p, C.c_int, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_int]
        self.lib = lib
        self.prob = prob
        g = space_group(prob.group_number)
        reps, _ = cosets(g.ops)
        self.keep = []

        def a(x, dt):
            x = np.ascontiguousarray(x, dtype=dt)
            self.keep.append(x)
            return x.ctypes.data

        p = PtProblem()
        p.nOps = len(g.ops)
        p.rot = a([o.r for o in g.ops], np.int32)
        p.trans = a([o.t_frac for o in g.ops], np.float64)
        p.nReps = len(reps)
        p.repRot = a([o.r for o in reps], np.int32)
        p.repTrans = a([o.t_frac for o in reps], np.float64)
        p.nAtoms = len(prob.atoms)
        p.pos = a([at['pos'] for at in prob.atoms], np.float64)
        p.wMult = a([at['mult'] / len(reps) for at in prob.atoms], np.float64)
        p.occ = a([at.get('occ', 1.0) for at in prob.atoms], np.float64)
        p.ffA = a([at['a'] for at in prob.atoms], np.float64)
        p.ffB = a([at['b'] for at in prob.atoms], np.float64)
        p.ffC = a([at['c'] for at in prob.atoms], np.float64)
        p.n = len(prob.tth)
        p.tth = a(prob.tth, np.float64)
        p.y = a(prob.y, np.float64)
        p.w = a(prob.w, np.float64)
        p.lambda1, p.lambda2, p.ratio, p.polK = prob.lambda1, prob.lambda2, prob.ratio, prob.pol_k
        p.minFwhm = prob.min_fwhm
        p.nBkg = prob.n_bkg
        p.dmin = 0.0 if dmin is None else float(dmin)
        po_dir = getattr(prob, 'po_dir', None)
        p.hasPo = 1 if po_dir is not None else 0
        if po_dir is not None:
            for i in range(3):
                p.poDir[i] = float(po_dir[i])
        p.hasAsym = 1 if getattr(prob, 'asym', False) else 0
        p.method = prob.method_code if hasattr(prob, 'method_code') else 0
        p.hasShift = 1 if getattr(prob, 'shift', False) else 0
        self.p = p

    def cost_full(self, v, with_pattern=False):
        v = np.ascontiguousarray(v, dtype=np.float64)
        y = np.zeros(len(self.prob.tth)) if with_pattern else None
        nr = C.c_int(0)
        c = self.lib.p6o_pt_cost(C.byref(self.p), v.ctypes.data, None if y is None else y.ctypes.data, C.byref(nr))
        return (c, y, nr.value) if with_pattern else c

    def cost(self, x):
        return self.cost_full(self.prob.apply(x))

    def pattern(self, prob, v):
        return self.cost_full(v, with_pattern=True)[1]

    def temper(self, x0, scales, chains=16, sweeps=50, max_temp=100.0, seed=12345, max_sweeps=0):
        prob = self.prob
        s = PtSetup()
        s.nv = len(x0)
        idx = np.ascontiguousarray(prob.index, dtype=np.int32)
        lo = np.ascontiguousarray(prob.lo, dtype=np.float64)
        hi = np.ascontiguousarray(prob.hi, dtype=np.float64)
        sc = np.ascontiguousarray(scales, dtype=np.float64)
        self.keep += [idx, lo, hi, sc]
        s.index, s.lo, s.hi, s.scales = idx.ctypes.data, lo.ctypes.data, hi.ctypes.data, sc.ctypes.data
        s.cubic = 1 if prob.system == 'cubic' else 0
        s.chains, s.sweeps, s.maxTemp, s.seed = chains, sweeps, max_temp, seed
        base = np.ascontiguousarray(prob.values, dtype=np.float64)
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        best = np.zeros(len(x0))
        stats = np.zeros(6)
        self.lib.p6o_pt_temper(C.byref(self.p), C.byref(s), base.ctypes.data, len(base), x0.ctypes.data,
                               best.ctypes.data, stats.ctypes.data, int(max_sweeps))
        return best, {'proposals': stats[0], 'accepted': stats[1], 'swapAttempts': stats[2], 'swaps': stats[3],
                      'bestChi2': stats[4], 'initialChi2': stats[5]}

    def _setup(self, scales=None):
        prob = self.prob
        s = PtSetup()
        s.nv = len(prob.refined)
        idx = np.ascontiguousarray(prob.index, dtype=np.int32)
        lo = np.ascontiguousarray(prob.lo, dtype=np.float64)
        hi = np.ascontiguousarray(prob.hi, dtype=np.float64)
        sc = np.ascontiguousarray(np.ones(s.nv) if scales is None else scales, dtype=np.float64)
        self.keep += [idx, lo, hi, sc]
        s.index, s.lo, s.hi, s.scales = idx.ctypes.data, lo.ctypes.data, hi.ctypes.data, sc.ctypes.data
        s.cubic = 1 if prob.system == 'cubic' else 0
        base = np.ascontiguousarray(prob.values, dtype=np.float64)
        self.keep.append(base)
        return s, base

    def normal(self, x):
        """normal() of the least-squares finish: (A = J'WJ, g = J'W r, f = chi^2) at x."""
        lib = self.lib
        lib.p6o_pt_normal.restype = C.c_int
        lib.p6o_pt_normal.argtypes = [C.POINTER(PtProblem), C.POINTER(PtSetup), C.c_void_p, C.c_int, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p]
        s, base = self._setup()
        nv = s.nv
        x = np.ascontiguousarray(x, dtype=np.float64)
        A = np.zeros((nv, nv))
        g = np.zeros(nv)
        f = C.c_double(0)
        ok = lib.p6o_pt_normal(C.byref(self.p), C.byref(s), base.ctypes.data, len(base), x.ctypes.data,
                               A.ctypes.data, g.ctypes.data, C.byref(f))
        if not ok:
            raise ValueError('the model is not finite at x')
        return A, g, f.value

    def lm(self, x0, max_iter=20, tol=1e-5):
        """lm() from x0: returns (x, {'chi2', 'iterations', 'accepted', 'code'})."""
        lib = self.lib
        lib.p6o_pt_lm.restype = C.c_int
        lib.p6o_pt_lm.argtypes = [C.POINTER(PtProblem), C.POINTER(PtSetup), C.c_void_p, C.c_int, C.c_void_p,
                                  C.c_int, C.c_double, C.c_void_p]
        s, base = self._setup()
        x = np.ascontiguousarray(np.array(x0, dtype=np.float64))
        out = np.zeros(4)
        lib.p6o_pt_lm(C.byref(self.p), C.byref(s), base.ctypes.data, len(base), x.ctypes.data, int(max_iter),
                      float(tol), out.ctypes.data)
        return x, {'chi2': out[0], 'iterations': int(out[1]), 'accepted': int(out[2]), 'code': int(out[3])}

    def linear_start(self, x):
        """One Gauss-Newton step on the scale and background parameters, kept if it
        lowers chi^2 (js/rietveld_core.js:2252-2263)."""
        prob = self.prob
        lin = [j for j, n in enumerate(prob.refined) if n == 'scale' or n.startswith('bkg')]
        A, g, f = self.normal(x)
        x = np.array(x, dtype=np.float64)
        if not lin:
            return x, f
        lib = self.lib
        lib.p6o_solve_spd.restype = C.c_int
        lib.p6o_solve_spd.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        M = np.ascontiguousarray(A[np.ix_(lin, lin)])
        rhs = np.ascontiguousarray(g[lin])
        d = np.zeros(len(lin))
        if lib.p6o_solve_spd(M.ctypes.data, rhs.ctypes.data, len(lin), d.ctypes.data):
            xt = x.copy()
            for a, q in enumerate(lin):
                xt[q] = min(prob.hi[q], max(prob.lo[q], x[q] + d[a]))
            ft = self.cost(xt)
            if ft < f:
                return xt, ft
        return x, f

    def rwp(self, chi2):
        """Rwp = sqrt(chi^2 / sum w y^2) over the points with w > 0 (datasetStats)."""
        w, y = self.prob.w, self.prob.y
        m = w > 0
        return float(np.sqrt(chi2 / np.sum(w[m] * y[m] ** 2)))


def contract_fp64(intensities, profile_t, yobs, w):
    """FP64 restatement of the fixed-profile pattern and its chi^2: y_calc =
    sum_k height_k col_k (evalPhase/render, js/rietveld_core.js:855-917) with
    the heights as the rows of ``intensities`` and the columns of the profile
    matrix (``profile_t`` is its transpose, points x reflections), and
    chi^2 = sum over w > 0 of w (y - y_calc)^2 (js/rietveld_core.js:1878-1889).
    Returns (Y, chi2)."""
    I = np.asarray(intensities, dtype=np.float64)
    Y = I @ np.asarray(profile_t, dtype=np.float64).T
    w = np.asarray(w, dtype=np.float64)
    m = w > 0
    r = np.asarray(yobs, dtype=np.float64)[None, :] - Y
    chi2 = (w[None, m] * r[:, m] ** 2).sum(axis=1)
    return Y, chi2


def profile_fitted_chi2(intensities, profile_t, yobs, w, n_active=None):
    """FP64 chi^2 of each row of ``intensities`` at its best scale:
    y_calc = s sum_k I_k col_k (evalPhase/render, js/rietveld_core.js:855-917)
    and chi^2(s) = sum over w > 0 of w (y - y_calc)^2 (:1878-1889), minimised
    over s >= 0 in closed form, s = sum w y Y / sum w Y^2.  Only the first
    ``n_active`` points count.  Returns (chi2, scale, sum w y^2)."""
    PT = np.asarray(profile_t, dtype=np.float64)
    n = PT.shape[0] if n_active is None else int(n_active)
    I = np.atleast_2d(np.asarray(intensities, dtype=np.float64))
    Y = I @ PT[:n].T
    ww = np.asarray(w, dtype=np.float64)[:n]
    ww = np.where(ww > 0, ww, 0.0)
    y = np.asarray(yobs, dtype=np.float64)[:n]
    syy = float((ww * y * y).sum())
    chi = np.empty(len(I))
    scale = np.zeros(len(I))
    for r in range(len(I)):
        a = float((ww * y * Y[r]).sum())
        b = float((ww * Y[r] * Y[r]).sum())
        if a > 0 and b > 0:
            scale[r] = a / b
            chi[r] = float((ww * (y - scale[r] * Y[r]) ** 2).sum())
        else:
            chi[r] = syy
    return chi, scale, syy


def wy_reflection_intensities(problem, A, x):
    """mult |F|^2 of every reflection (FP64) for the sites x (max_sites x 3
    fractional, already on their Wyckoff positions) of assignment A, from the
    packed tables: the per-reflection sums of swarm_reflection.wgsl's
    structure-factor pass before grouping."""
    atoms, _projs, _gm, hkl, mult, ftab = _refine_tables(problem, A)
    ms = problem.tables.max_sites
    x = np.asarray(x, dtype=np.float64).reshape(ms, 3)
    pos = np.array([(R @ x[s] + t) % 1.0 for s, R, t, _ in atoms])
    ty = np.array([a[3] for a in atoms])
    ph = 2 * np.pi * (hkl @ pos.T)
    f = ftab[:, ty]
    fr = (f * np.cos(ph)).sum(1)
    fi = (f * np.sin(ph)).sum(1)
    return mult * (fr * fr + fi * fi)


def mlp_unflatten(w, d_in, width, d_out):
    """W1 (d_in x width), b1, W2, b2, W3 (width x d_out), b3 from the flat FP32 block."""
    w = np.asarray(w, dtype=np.float64)
    sizes = [d_in * width, width, width * width, width, width * d_out, d_out]
    parts, o = [], 0
    for n in sizes:
        parts.append(w[o:o + n]); o += n
    W1, b1, W2, b2, W3, b3 = parts
    return W1.reshape(d_in, width), b1, W2.reshape(width, width), b2, W3.reshape(width, d_out), b3


def mlp_forward_fp64(w, X, d_in, width, d_out):
    """FP64 restatement of the proposal network: ReLU(X W1 + b1) -> ReLU(. W2 + b2) -> . W3 + b3."""
    W1, b1, W2, b2, W3, b3 = mlp_unflatten(w, d_in, width, d_out)
    H1 = np.maximum(np.asarray(X, np.float64) @ W1 + b1, 0)
    H2 = np.maximum(H1 @ W2 + b2, 0)
    return H2 @ W3 + b3, H1, H2


def mlp_grads_fp64(w, X, T, mask, d_in, width, d_out):
    """Gradient of the masked mean-squared error (1/n) sum mask (Y - T)^2 (0/1 masks), flat like w, and the loss."""
    X = np.asarray(X, np.float64)
    n = len(X)
    T = np.asarray(T, np.float64).reshape(n, d_out)
    M = np.ones_like(T) if mask is None else np.asarray(mask, np.float64).reshape(n, d_out)
    W1, b1, W2, b2, W3, b3 = mlp_unflatten(w, d_in, width, d_out)
    Y, H1, H2 = mlp_forward_fp64(w, X, d_in, width, d_out)
    E = (Y - T) * M
    loss = float((E * E).sum() / n)
    dY = 2 * E / n
    dW3 = H2.T @ dY
    db3 = dY.sum(0)
    dH2 = (dY @ W3.T) * (H2 > 0)
    dW2 = H1.T @ dH2
    db2 = dH2.sum(0)
    dH1 = (dH2 @ W2.T) * (H1 > 0)
    dW1 = X.T @ dH1
    db1 = dH1.sum(0)
    return np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3]), loss


# ---------------------------------------------------------------------------
# Wyckoff-constrained coordinate refinement (js/coord_refine.js:266-627), FP64
# ---------------------------------------------------------------------------
def _refine_tables(problem, A):
    """The images entering |F|^2 (site, R, t) of assignment A, the exact
    projectors, and the grouped observations, from the packed tables."""
    from fractions import Fraction
    T = problem.tables
    ms, nT = T.max_sites, T.n_tot
    gp = T.gen_pack[A * nT:(A + 1) * nT].astype(np.int64)
    sym = problem.sym_packed.astype(np.float64).reshape(-1, 12)

    def tfix(v):
        s = v * 24.0
        r = math.floor(s + 0.5)
        if abs(s - r) < 1e-4:
            return ((int(r) % 24) * 2 ** 32 + 12) // 24 / 2.0 ** 32
        f = v - math.floor(v)
        return (math.floor(f * 2 ** 32 + 0.5) % 2 ** 32) / 2.0 ** 32

    atoms = []
    for w in gp:
        if (w >> 24) & 1:
            continue
        site, op, ty = int(w & 0xFF), int((w >> 8) & 0xFFF), int(min((w >> 20) & 0xF, problem.n_elem - 1))
        R = sym[op, :9].round().reshape(3, 3)
        t = np.array([tfix(float(v)) for v in sym[op, 9:]])
        atoms.append((site, R, t, ty))
    projs = []
    sites = problem.assignments[A].sites
    for si in range(ms):
        if si < len(sites):
            Pm = np.array([float(Fraction(v)) for v in sites[si].w.P], dtype=np.float64).reshape(3, 3)
            Tv = np.array([tfix(float(Fraction(v))) for v in sites[si].w.T])
        else:
            Pm, Tv = np.zeros((3, 3)), np.zeros(3)
        projs.append((Pm, Tv))
    gm = problem.refl.group_meta.astype(np.float64).reshape(-1, 4)
    pk = problem.refl.refl_pack[0::2].astype(np.int64)
    hkl = np.stack([(pk & 0x3FF) - 512, ((pk >> 10) & 0x3FF) - 512, ((pk >> 20) & 0x3FF) - 512], 1).astype(np.float64)
    mult = problem.refl.refl_pack[1::2].astype(np.float64)
    ftab = problem.f_tab.astype(np.float64).reshape(-1, problem.n_elem)
    return atoms, projs, gm, hkl, mult, ftab


def wy_refine_intensities(problem, A, x, jac=False):
    """Ical per group (sum mult |F|^2) and, with jac, dIcal/du in the constrained space (P^T)."""
    atoms, projs, gm, hkl, mult, ftab = _refine_tables(problem, A)
    ms = problem.tables.max_sites
    x = np.asarray(x, dtype=np.float64).reshape(ms, 3)
    pos = np.array([(R @ x[s] + t) % 1.0 for s, R, t, _ in atoms])
    ty = np.array([a[3] for a in atoms])
    ical = np.zeros(len(gm))
    J = np.zeros((len(gm), ms * 3)) if jac else None
    for g, (r0, cnt, _, _) in enumerate(gm):
        grow = np.zeros(ms * 3)
        for r in range(int(r0), int(r0) + int(cnt)):
            ph = 2 * np.pi * (pos @ hkl[r])
            f = ftab[r, ty]
            c, s = np.cos(ph), np.sin(ph)
            a_, b_ = float((f * c).sum()), float((f * s).sum())
            ical[g] += mult[r] * (a_ * a_ + b_ * b_)
            if jac:
                w = mult[r] * 2 * 2 * np.pi * f * (b_ * c - a_ * s)
                for j, (site, R, _, _) in enumerate(atoms):
                    grow[3 * site:3 * site + 3] += w[j] * (R.T @ hkl[r])
        if jac:
            for si, (Pm, _) in enumerate(projs):
                J[g, 3 * si:3 * si + 3] = Pm.T @ grow[3 * si:3 * si + 3]
    return ical, J


def wy_refine(problem, A, x0, max_iter=60, lambda0=1e-3, lambda_up=10.0, lambda_down=0.4, lambda_max=1e8,
              tol_step=1e-6, tol_chi=1e-9, max_step=0.05):
    """refineCoordinatesAgainstWppf restated in FP64 on the packed tables:
    returns (coords, r_start, r_final, chi2, steps, converged)."""
    atoms, projs, gm, _, _, _ = _refine_tables(problem, A)
    ms = problem.tables.max_sites
    wt = np.where(gm[:, 3] > 0, gm[:, 3], 0.0)
    io = gm[:, 2]

    def project(x):
        x = x.reshape(ms, 3).copy()
        for si, (Pm, Tv) in enumerate(projs):
            x[si] = (Pm @ x[si] + Tv) % 1.0
        return x.reshape(-1)

    def scale_chi(ical):
        den = float((wt * ical * ical).sum())
        s = float((wt * io * ical).sum()) / den if den > 0 else 0.0
        return s, float((wt * (io - s * ical) ** 2).sum())

    oo = float((wt * io * io).sum())
    cur = project(np.asarray(x0, dtype=np.float64))
    ical, _ = wy_refine_intensities(problem, A, cur)
    s, chi = scale_chi(ical)
    r_start = math.sqrt(chi / oo)
    lam, steps, conv = lambda0, 0, False
    for _ in range(max_iter):
        ical, J = wy_refine_intensities(problem, A, cur, jac=True)
        s, chi = scale_chi(ical)
        Js = s * J
        res = io - s * ical
        JTr = (wt[:, None] * Js * res[:, None]).sum(0)
        JTJ = (Js * wt[:, None]).T @ Js
        stepped = False
        while lam < lambda_max:
            aug = JTJ.copy()
            dmax = float(np.max(np.diag(aug)))
            if not dmax > 0:
                conv = True
                break
            d = np.diag(aug).copy()
            aug[np.diag_indices_from(aug)] += lam * np.maximum(d, 1e-6 * dmax)
            try:
                L = np.linalg.cholesky(aug)
                dx = np.linalg.solve(L.T, np.linalg.solve(L, JTr))
            except np.linalg.LinAlgError:
                lam *= lambda_up
                continue
            dx = dx.reshape(ms, 3)
            for si, (Pm, _) in enumerate(projs):
                dx[si] = Pm @ dx[si]
            dx = dx.reshape(-1)
            big = float(np.max(np.abs(dx)))
            cap = max_step / big if big > max_step else 1.0
            trial = project(cur + cap * dx)
            itr, _ = wy_refine_intensities(problem, A, trial)
            s_tr, chi_tr = scale_chi(itr)
            if chi_tr < chi:
                moved = float(np.max(np.abs(trial - cur)))
                rel = (chi - chi_tr) / max(chi, 1e-300)
                cur, s, chi = trial, s_tr, chi_tr
                lam = max(lam * lambda_down, 1e-12)
                stepped, steps = True, steps + 1
                if moved < tol_step or rel < tol_chi:
                    conv = True
                break
            lam *= lambda_up
        if conv or not stepped:
            break
    ical, _ = wy_refine_intensities(problem, A, cur)
    s, chi = scale_chi(ical)
    return cur, r_start, math.sqrt(chi / oo), chi, steps, conv



# ---------------------------------------------------------------------------
# Rigid fragment with torsions -> fractional coordinates (FP64)
# ---------------------------------------------------------------------------
def _axis_angle_matrix(u, ang):
    """Rotation by ang about the unit axis u (Rodrigues' formula in matrix form)."""
    K = np.array([[0.0, -u[2], u[1]], [u[2], 0.0, -u[0]], [-u[1], u[0], 0.0]])
    return np.eye(3) + math.sin(ang) * K + (1.0 - math.cos(ang)) * (K @ K)


def fragment_coords_fp64(ref, axis_b, axis_c, moving, to_frac, params):
    """Fractional coordinates of a rigid fragment at parameters (t[3], q[4]
    = (w, x, y, z), torsion angles): torsion k turns the atoms in the bit mask
    moving[k] about the bond axis_b[k] -> axis_c[k] as the earlier torsions
    left it; then the rotation of the unit quaternion, the change of basis
    and the translation, wrapped into [0, 1).  The map the search uses for a
    molecule (direct-space parametrisation of js/molecule_rules.js)."""
    x = np.array(ref, dtype=np.float64).reshape(-1, 3).copy()
    p = np.asarray(params, dtype=np.float64)
    for k in range(len(axis_b)):
        b, c = x[axis_b[k]].copy(), x[axis_c[k]].copy()
        u = (c - b) / np.linalg.norm(c - b)
        Rk = _axis_angle_matrix(u, float(p[7 + k]))
        for i in range(len(x)):
            if (int(moving[k]) >> i) & 1:
                x[i] = b + Rk @ (x[i] - b)
    w, qx, qy, qz = p[3:7] / np.linalg.norm(p[3:7])
    # the quaternion's rotation as the composition of a turn by 2 acos(w) about (qx, qy, qz)
    s = math.sqrt(max(0.0, 1.0 - w * w))
    Rq = np.eye(3) if s < 1e-15 else _axis_angle_matrix(np.array([qx, qy, qz]) / s, 2.0 * math.atan2(s, w))
    f = (x @ Rq.T) @ np.asarray(to_frac, dtype=np.float64).reshape(3, 3).T + p[:3]
    return f - np.floor(f)
