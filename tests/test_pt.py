"""Parallel-tempering Rietveld model: the FP64 oracle against closed forms
restated from the reference's tests (tests/numerics.test.cjs:41-61,
186-200; tests/regressions.test.cjs:1583-1592), the synthetic NaCl workload,
and the CPU tempering schedule (js/rietveld_core.js:2171-2241)."""
import ctypes as C
import math

import numpy as np
import pytest

from powder6_b200.pt_gpu import (PTContext, compile, nacl_problem, natural_scales, pt_scales, reflection_dmin,
                                 start_vectors, synthesise)


@pytest.fixture(scope='module')
def nacl(oracle):
    P = nacl_problem(seed=1)
    M = oracle.PtModel(P)
    truth = synthesise(P, M.pattern, seed=1)
    return P, oracle.PtModel(P, dmin=reflection_dmin(P)), truth


def hooks(oracle):
    lib = oracle.load()
    for name in ('p6o_lp', 'p6o_peak_fwhm', 'p6o_soft_positive', 'p6o_soft_floor'):
        getattr(lib, name).restype = C.c_double
        getattr(lib, name).argtypes = [C.c_double, C.c_double]
    lib.p6o_voigt_raw.restype = C.c_double
    lib.p6o_voigt_raw.argtypes = [C.c_double] * 4
    lib.p6o_prepare_tch.restype = None
    lib.p6o_prepare_tch.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_void_p]
    return lib


def test_lorentz_polarisation_closed_forms(oracle):
    lib = hooks(oracle)
    assert abs(lib.p6o_lp(90, 1) - 0.5 / (0.5 * math.sqrt(0.5))) < 1e-12
    assert lib.p6o_lp(0, 1) == 1 and lib.p6o_lp(180, 1) == 1          # degenerate geometry leaves intensity alone
    t = 60.0
    L = 1 / (math.sin(math.radians(30)) ** 2 * math.cos(math.radians(30)))
    assert abs(lib.p6o_lp(t, 0) - L) < 1e-12                           # K = 0: no polarisation
    assert abs(lib.p6o_lp(t, 1) - L * (1 + 0.25) / 2) < 1e-12


def test_width_helpers(oracle):
    lib = hooks(oracle)
    assert abs(lib.p6o_peak_fwhm(0.1, 1e-12) - 0.1) < 1e-9              # pure Gaussian
    assert abs(lib.p6o_peak_fwhm(1e-12, 0.1) - 0.1) < 1e-9              # pure Lorentzian
    assert lib.p6o_peak_fwhm(0.1, 0.1) > 0.1
    assert lib.p6o_soft_positive(0.0, 0.3) == pytest.approx(0.3)        # f at x = 0
    assert lib.p6o_soft_positive(1e6, 0.3) == pytest.approx(1e6)
    assert lib.p6o_soft_positive(-1e6, 0.3) == pytest.approx(0.09 / 1e6, rel=1e-6)
    assert lib.p6o_soft_floor(0.0, 0.04) == 0.04 and lib.p6o_soft_floor(2.0, 0.04) == 2.0
    assert abs(lib.p6o_soft_floor(0.1, 0.04) - 0.1) / 0.1 < 0.01      # within 1 % of x by 2.5 f


def test_area_normaliser_matches_the_integral(oracle):
    """The analytic area of the unit-height pseudo-Voigt equals its integral
    (the regressions.test.cjs:1583-1592 check, without asymmetry)."""
    lib = hooks(oracle)
    v = np.zeros(14)
    v[7:12] = [7.2136, -3.6068, 5.4102, 1.0, 2.0]
    out = np.zeros(7)
    lib.p6o_prepare_tch(v.ctypes.data, 0.04, 60.0, out.ctypes.data)
    inv, cL, cG, area = out[1], out[2], out[3], out[6]
    fwhm = 1 / inv
    L, n = 3000 * fwhm, 400000
    u = -1 + (np.arange(n) + 0.5) * 2 / n
    x = L * u ** 3
    dx = 3 * L * u * u * 2 / n
    vals = np.array([lib.p6o_voigt_raw(float(d), inv, cL, cG) for d in x[::50]])
    integral = float((vals * dx[::50] * 50).sum())
    assert abs(integral - area) < 2e-4 * area
    # unit height at the centre, and the pedestal is the edge value
    assert abs(lib.p6o_voigt_raw(0.0, inv, cL, cG) - 1.0) < 1e-12
    assert abs(out[4] - lib.p6o_voigt_raw(out[5], inv, cL, cG)) < 1e-15


def test_synthetic_nacl_and_chi2_at_truth(nacl):
    P, M, truth = nacl
    assert len(P.tth) == 5501 and P.tth[0] == 10.0 and abs(P.tth[-1] - 120.0) < 1e-9
    c, y, nr = M.cost_full(P.values, True)
    assert nr == 18
    n = len(P.tth)
    assert abs(c - n) < 6 * math.sqrt(2 * n)            # Poisson counts, w = 1/y: chi^2 ~ n
    assert 0.9e4 < P.y.max() < 1.1e4
    for x in start_vectors(P, truth, 4, seed=3):
        assert M.cost(x) > 2 * c                         # +/-5 % starts are far off


def test_plan_envelope_and_dmin(nacl):
    P, M, truth = nacl
    plan = compile(PTContext(P, truth, {'chains': 64, 'sweeps': 10, 'maxTemp': 100.0, 'seed': 1,
                                        'scales': natural_scales(P, truth)}))
    assert plan.reflection_count >= 18 and plan.stride == 3 * 7 + 12
    # dmin from 2theta_max 120 + the 10 deg window + |zero| bound (0.1)
    assert abs(plan.dmin - 1.5406 / (2 * math.sin(math.radians(130.101) / 2))) < 1e-9


def test_cpu_tempering_schedule_and_determinism(nacl):
    """Proposals = chains x sweeps x nv (webgpu-pt.js:131-136); same seed, same run."""
    P, M, truth = nacl
    x0 = start_vectors(P, truth, 1, seed=5)[0]
    sc = pt_scales(P, x0)
    b1, s1 = M.temper(x0, sc, chains=4, sweeps=10, seed=99)
    b2, s2 = M.temper(x0, sc, chains=4, sweeps=10, seed=99)
    assert np.array_equal(b1, b2) and s1 == s2
    assert s1['proposals'] == 4 * 10 * 7
    assert s1['swapAttempts'] == 5 * 2 + 5 * 1                # even sweeps 2 pairs, odd sweeps 1 pair
    assert s1['bestChi2'] <= s1['initialChi2']


def test_normal_equations_are_consistent(nacl):
    """A = J'WJ is symmetric positive semi-definite; f is the chi^2; g = J'W r
    is minus half the gradient of chi^2 (checked along the Gauss-Newton direction)."""
    P, M, truth = nacl
    x = truth.copy()
    x[1] *= 1.0005
    A, g, f = M.normal(x)
    assert np.allclose(A, A.T, rtol=0, atol=0)
    assert abs(f - M.cost(x)) <= 1e-12 * f
    assert np.all(np.linalg.eigvalsh(A / np.sqrt(np.outer(np.diag(A), np.diag(A)))) > -1e-9)
    d = np.linalg.solve(A, g)
    t = 1e-4
    slope = (M.cost(x + t * d) - M.cost(x - t * d)) / (2 * t)
    assert abs(slope + 2 * g @ d) < 1e-4 * abs(2 * g @ d)


def test_lm_converges_from_near_the_truth(nacl):
    """The least-squares finish from a start inside the basin reaches chi^2 ~ n
    (Poisson counts, w = 1/y) and stops on the chi^2-change criterion."""
    P, M, truth = nacl
    x0 = truth.copy()
    x0[1] *= 1.001
    x0[3] *= 1.2
    x, info = M.lm(x0, 30)
    n = len(P.tth)
    assert info['code'] in (1, 2)
    assert abs(info['chi2'] - n) < 6 * math.sqrt(2 * n)
    assert info['chi2'] <= M.cost(truth) + 1e-9
    assert abs(x[1] - truth[1]) < 1e-4


def test_linear_start_solves_the_scale(nacl):
    """With every other parameter at the truth, one Gauss-Newton step on the
    (linear) scale recovers it."""
    P, M, truth = nacl
    x0 = truth.copy()
    x0[0] *= 1.3
    x, f = M.linear_start(x0)
    assert abs(x[0] - truth[0]) < 1e-3 * truth[0]
    assert f < M.cost(x0)


# ---------------------------------------------------------------------------
# March-Dollase preferred orientation (js/rietveld_core.js:824-853)
# ---------------------------------------------------------------------------
def _po_lib(oracle):
    lib = oracle.load()
    lib.p6o_po_factor.restype = C.c_double
    lib.p6o_po_factor.argtypes = [C.POINTER(oracle.PtProblem), C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int]
    return lib


def _po_restated(cell, rots, h, d, r):
    """Independent restatement: the reciprocal metric as the inverse of the
    direct metric, equivalents h R without duplicates, the mean of
    (r^2 c^2 + (1 - c^2) / r)^(-3/2)."""
    a, b, c, al, be, ga = cell
    ca, cb, cg = (math.cos(math.radians(t)) for t in (al, be, ga))
    G = np.array([[a * a, a * b * cg, a * c * cb], [a * b * cg, b * b, b * c * ca], [a * c * cb, b * c * ca, c * c]])
    Gs = np.linalg.inv(G)
    eqs = {tuple(int(v) for v in np.asarray(h) @ np.asarray(R).reshape(3, 3)) for R in rots}
    d = np.asarray(d, dtype=np.float64)
    vals = []
    for e in eqs:
        e = np.asarray(e, dtype=np.float64)
        cos = (e @ Gs @ d) / math.sqrt((e @ Gs @ e) * (d @ Gs @ d))
        c2 = min(1.0, cos * cos)
        vals.append((r * r * c2 + (1 - c2) / r) ** -1.5)
    return float(np.mean(vals))


def test_march_dollase_factor_closed_form_and_restatement(oracle):
    """Cubic (002) along [001]: two equivalents parallel, four perpendicular,
    so the factor is (2 r^-3 + 4 r^1.5) / 6; r = 1 gives 1; a monoclinic cell
    (P2_1/c, beta = 104 deg) against the restatement with the inverse metric."""
    from powder6_b200.pt_gpu import with_preferred_orientation
    from powder6_b200.symmetry import space_group
    lib = _po_lib(oracle)
    P = with_preferred_orientation(nacl_problem(seed=1), (0, 0, 1), 0.7)
    M = oracle.PtModel(P)
    cub = np.array([5.64, 5.64, 5.64, 90.0, 90.0, 90.0])
    for r in (0.6, 0.85, 1.0, 1.4):
        got = lib.p6o_po_factor(C.byref(M.p), cub.ctypes.data, r, 0, 0, 2)
        assert abs(got - (2 * r ** -3 + 4 * r ** 1.5) / 6) < 1e-13
    assert lib.p6o_po_factor(C.byref(M.p), cub.ctypes.data, 1.0, 1, 1, 1) == 1.0
    P14 = with_preferred_orientation(nacl_problem(seed=1), (1, 0, 2), 0.8)
    P14.group_number = 14
    M14 = oracle.PtModel(P14)
    rots = [o.r for o in space_group(14).ops]
    mono = np.array([7.1, 9.3, 11.2, 90.0, 104.0, 90.0])
    for hkl in ((1, 0, 0), (1, 2, 3), (-2, 1, 1), (0, 4, 1)):
        for r in (0.55, 0.8, 1.3):
            got = lib.p6o_po_factor(C.byref(M14.p), mono.ctypes.data, r, *hkl)
            want = _po_restated(mono, rots, hkl, (1, 0, 2), r)
            assert abs(got - want) < 1e-12 * want, (hkl, r, got, want)


def test_march_dollase_cost_reduces_to_plain_at_r_one(nacl, oracle):
    """r = 1 multiplies every height by exactly 1; r != 1 changes chi^2."""
    from powder6_b200.pt_gpu import with_preferred_orientation
    P, M, truth = nacl
    Pp = with_preferred_orientation(P, (0, 0, 1), 1.0)
    Mp = oracle.PtModel(Pp, dmin=reflection_dmin(P))
    assert Mp.cost(np.append(truth, 1.0)) == M.cost(truth)
    assert Mp.cost(np.append(truth, 0.8)) > 1.1 * M.cost(truth)


# ---------------------------------------------------------------------------
# SL/HL asymmetry (js/profile.js:608-617, :737-740, :799-826)
# ---------------------------------------------------------------------------
def _raw_asym(delta, inv, cL, cG, asym):
    """evalVoigt of the TCH shape, untruncated and without pedestal, restated."""
    d = np.asarray(delta, dtype=np.float64)
    if asym != 0:
        t = np.clip(asym * d, -0.95, 0.95)
        d = np.where(np.abs(d) >= 1e-9, d / (1.0 - t), d)
    dg = (d * inv) ** 2
    return cL / (1 + 4 * dg) + cG * np.exp(-2.772588722239781 * dg)


def test_asymmetry_area_matches_the_brute_force_integral(oracle):
    """The regressions.test.cjs:1583-1592 check: U = V = 0, W = X = 5, Y = 0,
    SL = 0.05, HL = 0.02, minFwhm 0.005 at 2theta = 10: the area with the
    asymmetry's correction equals the analytic area plus the brute-force
    integral of (asymmetric - symmetric) within 2e-4, and differs from the
    analytic area by more than 1 %."""
    lib = oracle.load()
    lib.p6o_prepare_tch_asym.restype = None
    lib.p6o_prepare_tch_asym.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_void_p]
    lib.p6o_prepare_tch.restype = None
    lib.p6o_prepare_tch.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_void_p]
    v = np.zeros(14)
    v[7:12] = [0.0, 0.0, 5.0, 5.0, 0.0]
    out = np.zeros(8)
    lib.p6o_prepare_tch_asym(v.ctypes.data, 0.005, 10.0, 0.05, 0.02, out.ctypes.data)
    sym = np.zeros(7)
    lib.p6o_prepare_tch(v.ctypes.data, 0.005, 10.0, sym.ctypes.data)
    inv, cL, cG, area, asym = out[1], out[2], out[3], out[6], out[7]
    assert abs(asym - (0.05 / math.tan(math.radians(5.0)) + 0.02)) < 1e-12
    assert abs(out[5] - min(10.0, 2 * sym[5])) < 1e-12 or out[5] == 10.0       # the window doubles
    analytic = sym[6]
    L, n = 3000 / inv, 200000
    u = -1 + (np.arange(n) + 0.5) * 2 / n
    x = L * u ** 3
    dx = 3 * L * u * u * 2 / n
    diff = float(((_raw_asym(x, inv, cL, cG, asym) - _raw_asym(x, inv, cL, cG, 0.0)) * dx).sum())
    assert abs(area - (analytic + diff)) < 2e-4 * (analytic + diff), (area, analytic + diff)
    assert area > 1.01 * analytic


def test_asymmetry_cost_reduces_to_symmetric_at_zero(nacl, oracle):
    """SL = HL = 0 leaves every peak symmetric: the same chi^2 bit for bit."""
    from powder6_b200.pt_gpu import with_asymmetry
    P, M, truth = nacl
    Pa = with_asymmetry(P, 0.0, 0.0)
    Ma = oracle.PtModel(Pa, dmin=reflection_dmin(P))
    assert Ma.cost(np.append(truth, [0.0, 0.0])) == M.cost(truth)
    assert Ma.cost(np.append(truth, [0.2, 0.05])) > 1.05 * M.cost(truth)


# ---------------------------------------------------------------------------
# WPPF / Le Bail free intensities (js/pt_gpu.js:259-297)
# ---------------------------------------------------------------------------
def _nnls_lib(oracle):
    lib = oracle.load()
    lib.p6o_nnls_normal.restype = C.c_int
    lib.p6o_nnls_normal.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    return lib


def test_nnls_on_normal_equations_matches_scipy(oracle):
    """The oracle's Lawson-Hanson solve on H = A^T A, rhs = A^T b reaches
    scipy's NNLS optimum of |A x - b| (relative excess below 1e-12), on random
    problems of 1..40 columns, a third of them with two nearly collinear
    columns, and on the degenerate cases: all-negative rhs (x = 0) and one
    column."""
    from scipy.optimize import nnls
    lib = _nnls_lib(oracle)
    rng = np.random.default_rng(0)
    for t in range(120):
        m = int(rng.integers(1, 41))
        A = rng.normal(size=(int(rng.integers(m, 3 * m + 5)), m))
        b = 3 * rng.normal(size=A.shape[0])
        if t % 3 == 0 and m > 1:
            A[:, 0] = 0.999 * A[:, 1] + 1e-3 * A[:, 0]
        xs, _ = nnls(A, b, maxiter=10000)
        H, r, x = np.ascontiguousarray(A.T @ A), np.ascontiguousarray(A.T @ b), np.zeros(m)
        assert lib.p6o_nnls_normal(H.ctypes.data, r.ctypes.data, m, x.ctypes.data) >= 0
        assert np.all(x >= 0)
        fs, fo = np.sum((A @ xs - b) ** 2), np.sum((A @ x - b) ** 2)
        assert fo - fs <= 1e-12 * max(fs, 1.0), (t, fo, fs)
    A = np.abs(rng.normal(size=(12, 5)))
    H, r, x = np.ascontiguousarray(A.T @ A), np.ascontiguousarray(-A.T @ np.ones(12)), np.ones(5)
    lib.p6o_nnls_normal(H.ctypes.data, r.ctypes.data, 5, x.ctypes.data)
    assert np.all(x == 0)
    H, r, x = np.array([[4.0]]), np.array([2.0]), np.zeros(1)
    lib.p6o_nnls_normal(H.ctypes.data, r.ctypes.data, 1, x.ctypes.data)
    assert x[0] == 0.5


def _free(P, method='wppf'):
    import copy
    out = copy.copy(P)
    out.method = method
    return out


def test_free_intensity_cost_bounds_and_invariances(nacl, oracle):
    """A free-intensity fit is never worse than the Rietveld heights, which
    are one non-negative choice of the same columns: chi^2(wppf) <= chi^2
    (rietveld) at the truth and at start vectors.  At the truth it sits at the
    noise level (about one per point).  The scale and Biso do not enter it
    (bit-identical chi^2), 'lebail' and 'wppf' are the same fit, and any other
    method name is rejected."""
    P, M, truth = nacl
    Pw = _free(P)
    Mw = oracle.PtModel(Pw, dmin=reflection_dmin(P))
    for x in [truth] + start_vectors(P, truth, 6, seed=21):
        assert Mw.cost(x) <= M.cost(x) * (1 + 1e-12)
    c = Mw.cost(truth)
    assert 0.8 * len(P.tth) < c < 1.2 * len(P.tth)
    x = truth.copy()
    x[P.refined.index('scale')] *= 1.3
    x[P.refined.index('Biso')] += 0.7
    assert Mw.cost(x) == c
    assert oracle.PtModel(_free(P, 'lebail'), dmin=reflection_dmin(P)).cost(truth) == c
    with pytest.raises(ValueError):
        _free(P, 'pawley').method_code


def test_free_intensity_pattern_is_the_nnls_fit(nacl, oracle):
    """The free-intensity pattern returned with chi^2 is consistent with it
    (chi^2 = sum w (y - ycalc)^2 to 1e-9), its peak part (ycalc minus the
    background) is non-negative everywhere, and it lowers chi^2 below the
    background alone.  The background is the Rietveld pattern at scale 0."""
    P, M, truth = nacl
    Mw = oracle.PtModel(_free(P), dmin=reflection_dmin(P))
    x = start_vectors(P, truth, 1, seed=5)[0]
    v = P.apply(x)
    c, y, _ = Mw.cost_full(v, True)
    bk_only = v.copy()
    bk_only[0] = 0.0
    _, bkg, _ = M.cost_full(bk_only, True)
    w = P.w
    r = P.y - y
    assert abs(c - np.sum(w * r * r)) <= 1e-9 * c
    # every heights-and-background decomposition: the fitted peaks are y - bkg
    peaks = y - bkg
    assert np.min(peaks) >= -1e-9 * np.max(np.abs(peaks))
    # the fit lowers chi^2 from the background alone
    assert c < np.sum(w * (P.y - bkg) ** 2)


# ---------------------------------------------------------------------------
# Sample displacement and transparency (js/pt_gpu.js:169-171, :355)
# ---------------------------------------------------------------------------
def test_sample_shift_reduces_to_plain_at_zero(nacl, oracle):
    """disp = transp = 0 leaves every peak where it was: the same chi^2 bit
    for bit; a displacement of 100 moves them."""
    from powder6_b200.pt_gpu import with_sample_shift
    P, M, truth = nacl
    Ps = with_sample_shift(P, 0.0, 0.0)
    Ms = oracle.PtModel(Ps, dmin=reflection_dmin(P))
    assert Ms.cost(np.append(truth, [0.0, 0.0])) == M.cost(truth)
    assert Ms.cost(np.append(truth, [100.0, 0.0])) > 1.05 * M.cost(truth)


def test_sample_shift_is_a_local_zero_point(nacl, oracle):
    """Near one isolated peak, displacement and transparency act as the zero
    point (-disp 1e-3 cos(theta) + transp sin(2 theta)) in degrees at that
    peak's Bragg angle: with the doublet off, the (200) peak of the shifted
    pattern matches the unshifted one with that zero point to 2e-3 of its
    height within +-0.3 degrees."""
    import copy
    from powder6_b200.pt_gpu import with_sample_shift
    P, _, truth = nacl
    P1 = copy.copy(P)
    P1.ratio = 0.0
    disp, transp = 60.0, 0.003
    Ps = with_sample_shift(P1, disp, transp)
    v = P1.apply(truth)
    a = v[1]
    bragg = 2 * math.degrees(math.asin(P1.lambda1 * 2 / (2 * a)))       # (200): d = a / 2
    th = math.radians(bragg / 2)
    dz = (-disp * 1e-3 * math.cos(th) + transp * math.sin(2 * th)) * 180 / math.pi
    ys = oracle.PtModel(Ps, dmin=reflection_dmin(Ps)).cost_full(np.append(v, [disp, transp]), True)[1]
    vz = v.copy()
    vz[P1.full_index('zero')] += dz
    yz = oracle.PtModel(P1, dmin=reflection_dmin(Ps)).cost_full(vz, True)[1]
    sel = np.abs(P1.tth - (bragg + dz)) < 0.3
    assert abs(dz) > 0.05
    assert np.max(np.abs(ys[sel] - yz[sel])) <= 2e-3 * np.max(yz[sel])
