"""Parallel-tempering backend on the B200 against the FP64 oracle.

The kernel computes the per-reflection work (|F|^2, TCH widths, areas, Lp,
doublet weight) and the chi^2 accumulation in FP64 and the per-point profile
shape in FP32, as the reference's WGSL kernel does in FP32 throughout
(js/pt_gpu.js:229-369).  Tolerances: chi^2 relative 2e-6, calculated
pattern absolute 2e-5 of the pattern maximum.  run() itself applies the
reference's 1e-3 validation gate (js/pt_gpu.js:413-415)."""
import math

import numpy as np
import pytest

from powder6_b200.pt_gpu import (PTContext, PTSession, nacl_problem, pt_scales, reflection_dmin, run, start_vectors,
                                 synthesise)

pytestmark = pytest.mark.gpu

CHI2_RTOL = 1e-6
PATTERN_ATOL_FRAC = 2e-5


@pytest.fixture(scope='module')
def nacl(oracle):
    P = nacl_problem(seed=1)
    truth = synthesise(P, oracle.PtModel(P).pattern, seed=1)
    return P, oracle.PtModel(P, dmin=reflection_dmin(P)), truth


def ctx_of(P, x0, chains=16, sweeps=20, seed=7, max_temp=100.0, cost=None):
    return PTContext(P, x0, {'chains': chains, 'sweeps': sweeps, 'maxTemp': max_temp, 'seed': seed,
                             'scales': pt_scales(P, x0)}, cost=cost)


def test_costs_match_oracle(nacl):
    P, M, truth = nacl
    xs = [truth] + start_vectors(P, truth, 7, seed=11)
    with PTSession(ctx_of(P, truth, chains=len(xs))) as s:
        g = s.costs(xs)
    for x, gc in zip(xs, g):
        c = M.cost(x)
        assert abs(gc - c) <= CHI2_RTOL * c, (gc, c)


def test_pattern_matches_oracle(nacl):
    P, M, truth = nacl
    xs = [truth] + start_vectors(P, truth, 3, seed=12)
    with PTSession(ctx_of(P, truth, chains=4)) as s:
        _, ys = s.costs(xs, with_pattern=True)
    for x, y in zip(xs, ys):
        _, yo, _ = M.cost_full(P.apply(x), True)
        assert np.max(np.abs(y - yo)) <= PATTERN_ATOL_FRAC * np.max(np.abs(yo))


def test_out_of_envelope_cell_is_infinite_or_consistent(nacl):
    """A cell inside the bounds always scores finitely; a degenerate one (a = 0) is +inf."""
    P, M, truth = nacl
    x = truth.copy()
    x[1] = P.hi[1]
    bad = truth.copy()
    bad[1] = 0.0
    with PTSession(ctx_of(P, truth, chains=2)) as s:
        g = s.costs([x, bad])
    assert abs(g[0] - M.cost(x)) <= CHI2_RTOL * M.cost(x)
    assert math.isinf(g[1])


def test_batch_counters_and_monotone_best(nacl):
    P, M, truth = nacl
    x0 = start_vectors(P, truth, 1, seed=5)[0]
    chains, sweeps = 16, 12
    with PTSession(ctx_of(P, x0, chains=chains)) as s:
        s.initial([x0])
        s.batch(1, True)
        _, _, c0, _ = s.exact_state()
        s.batch(sweeps)
        x, best, costs, counters = s.exact_state()
        st = s.state()
        launches = s.launch_count()
    nv = len(x0)
    assert counters[:, 1].sum() == chains * sweeps * nv                 # proposals; the bootstrap sweep counts none
    assert np.all(counters[:, 0] <= counters[:, 1])                    # accepted <= proposals
    assert np.all(counters[:, 2] <= counters[:, 3])                    # swaps <= attempts
    assert np.all(costs[:, 1] <= c0[:, 1] + 1e-9)                       # best never worsens
    for c in range(chains):                                             # each best re-scores to its cost
        assert abs(M.cost(best[c]) - costs[c, 1]) <= CHI2_RTOL * costs[c, 1]
        assert np.all(best[c] >= P.lo - 1e-12) and np.all(best[c] <= P.hi + 1e-12)
    stride = 3 * nv + 12
    assert st.shape == (chains * stride,)
    assert np.allclose(st.reshape(chains, stride)[:, :nv], x, rtol=1e-6, atol=1e-6)
    assert launches >= sweeps + 1


def test_two_cta_clusters_match_one_cta_chains(nacl):
    """Sixteen chains leave most SMs idle, so the session sweeps each chain on
    a two-CTA cluster.  The bootstrap chi^2 matches the cost kernel's to 1e-13
    in both splits, and ten sweeps make the same Metropolis decisions: the
    splits differ only in the order of the chi^2 sum."""
    P, M, truth = nacl
    xs = start_vectors(P, truth, 16, seed=21)
    runs = {}
    for split in (2, 1):
        with PTSession(ctx_of(P, truth, chains=16, seed=4)) as s:
            if split == 2:
                assert s.split == 2
            s.split = split
            ref = np.array(s.costs(xs))
            s.initial(xs)
            s.batch(1, True)
            _, _, c0, _ = s.exact_state()
            assert np.max(np.abs(c0[:, 0] - ref) / ref) < 1e-13
            s.batch(10)
            runs[split] = s.exact_state()
    x2, b2, c2, n2 = runs[2]
    x1, b1, c1, n1 = runs[1]
    assert np.array_equal(n2, n1)
    assert np.allclose(x2, x1, rtol=1e-12, atol=0) and np.allclose(c2, c1, rtol=1e-12, atol=0)


def test_determinism(nacl):
    P, M, truth = nacl
    x0 = start_vectors(P, truth, 1, seed=6)[0]
    out = []
    for _ in range(2):
        with PTSession(ctx_of(P, x0, chains=8, seed=3)) as s:
            s.initial([x0])
            s.batch(1, True)
            s.batch(5)
            out.append(s.exact_state())
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_run_reduces_chi2_and_validates(nacl):
    P, M, truth = nacl
    x0 = start_vectors(P, truth, 1, seed=8)[0]
    c0 = M.cost(x0)
    ctx = ctx_of(P, x0, chains=32, sweeps=40, cost=M.cost)
    ctx.setup['initialCost'] = c0
    r = run(ctx)
    assert r['pt']['validationError'] < 1e-5
    assert r['pt']['bestChi2'] < 0.5 * c0
    assert abs(M.cost(r['x']) - r['pt']['bestChi2']) <= 1e-12 * c0
    assert r['pt']['proposals'] == 32 * 40 * len(x0)


def test_run_rejects_a_disagreeing_cost(nacl):
    P, M, truth = nacl
    x0 = start_vectors(P, truth, 1, seed=9)[0]
    ctx = ctx_of(P, x0, chains=4, sweeps=2, cost=lambda x: 1.01 * M.cost(x))
    with pytest.raises(RuntimeError, match='disagrees'):
        run(ctx)


def near_truth(truth):
    x0 = truth.copy()
    x0[1] *= 1.001
    x0[3] *= 1.2
    return x0


def test_fp64_model_and_normal_equations_match_oracle(nacl):
    """FP64 model cost, A = J'WJ, g = J'W r and f against the oracle.  A and g
    are compared on their natural scales sqrt(A_ii A_jj) and sqrt(A_ii f)."""
    P, M, truth = nacl
    x = near_truth(truth)
    with PTSession(ctx_of(P, truth, chains=2)) as s:
        c = s.model_costs([x, truth])
        A, g, f = s.normal(x)
    assert abs(c[0] - M.cost(x)) <= 1e-10 * c[0]
    assert abs(c[1] - M.cost(truth)) <= 1e-10 * c[1]
    Ao, go, fo = M.normal(x)
    assert abs(f - fo) <= 1e-10 * fo
    d = np.sqrt(np.diag(Ao))
    assert np.max(np.abs(A - Ao) / np.outer(d, d)) < 1e-7
    assert np.max(np.abs(g - go) / (d * math.sqrt(fo))) < 1e-7


def test_linear_start_matches_oracle(nacl):
    P, M, truth = nacl
    x0 = truth.copy()
    x0[0] *= 1.3
    with PTSession(ctx_of(P, truth, chains=2)) as s:
        xg, fg = s.linear_start(x0)
    xo, fo = M.linear_start(x0)
    assert np.allclose(xg, xo, rtol=1e-9, atol=0)
    assert abs(fg - fo) <= 1e-9 * fo


def test_lm_finish_matches_oracle(nacl):
    P, M, truth = nacl
    x0 = near_truth(truth)
    with PTSession(ctx_of(P, truth, chains=2)) as s:
        xg, ig = s.lm(x0, 30)
    xo, io = M.lm(x0, 30)
    assert ig['code'] == io['code'] and ig['accepted'] == io['accepted']
    assert abs(ig['chi2'] - io['chi2']) <= 1e-9 * io['chi2']
    assert np.allclose(xg, xo, rtol=1e-7, atol=1e-9)


def test_refine_reaches_the_target_rwp(nacl):
    """Linear start, tempering and the least-squares finish on the device from a
    +/-5 % start reach Rwp <= 1.05 x the Rwp of the finish started at the truth."""
    from powder6_b200.pt_gpu import refine, rwp
    P, M, truth = nacl
    _, ref = M.lm(truth, 30)
    target = 1.05 * rwp(P, ref['chi2'])
    x0 = start_vectors(P, truth, 1, seed=8)[0]
    ctx = ctx_of(P, x0, chains=64, sweeps=300)
    r = refine(ctx, target_chi2=target ** 2 * float(np.sum(P.w * P.y ** 2)))
    assert r['rwp'] <= target
    assert r['time_to_target'] is not None and r['time_to_target'] <= r['seconds']['lm']
    assert abs(M.cost(r['x']) - r['chi2']) <= 1e-9 * r['chi2']


# ---------------------------------------------------------------------------
# March-Dollase preferred orientation (js/rietveld_core.js:824-853), refined
# ---------------------------------------------------------------------------
@pytest.fixture(scope='module')
def nacl_po(nacl, oracle):
    from powder6_b200.pt_gpu import with_preferred_orientation
    P, M, truth = nacl
    Pp = with_preferred_orientation(P, (1, 1, 0), 1.0, lo=0.5, hi=2.0)
    return Pp, oracle.PtModel(Pp, dmin=reflection_dmin(Pp)), np.append(truth, 0.8)


def test_preferred_orientation_costs_match_oracle(nacl_po):
    """chi^2 with the March-Dollase factor (lanes over the equivalents, FP64)
    within the tempering cost's 2e-6, at r = 0.6 .. 1.6 along [110]."""
    P, M, x0 = nacl_po
    xs = [x0] + [np.append(v[:-1], r) for v, r in zip(start_vectors(P, x0, 4, seed=21), (0.6, 1.0, 1.25, 1.6))]
    with PTSession(ctx_of(P, x0, chains=len(xs))) as s:
        g = s.costs(xs)
        c64 = s.model_costs(xs)
    for x, gc, gm in zip(xs, g, c64):
        c = M.cost(x)
        assert abs(gc - c) <= CHI2_RTOL * c, (gc, c)
        assert abs(gm - c) <= 1e-10 * c, (gm, c)


def test_preferred_orientation_normal_equations_and_lm_match_oracle(nacl_po):
    """The r column is the reference's forward difference; A, g, f and an LM
    run from r = 0.8 match the oracle as the other parameters do."""
    P, M, x0 = nacl_po
    x = near_truth(x0)
    with PTSession(ctx_of(P, x0, chains=2)) as s:
        A, g, f = s.normal(x)
        xg, ig = s.lm(x, 30)
    Ao, go, fo = M.normal(x)
    assert abs(f - fo) <= 1e-10 * fo
    d = np.sqrt(np.diag(Ao))
    assert d[-1] > 0
    assert np.max(np.abs(A - Ao) / np.outer(d, d)) < 1e-7
    assert np.max(np.abs(g - go) / (d * math.sqrt(fo))) < 1e-7
    xo, io = M.lm(x, 30)
    assert ig['code'] == io['code'] and ig['accepted'] == io['accepted']
    assert abs(ig['chi2'] - io['chi2']) <= 1e-9 * io['chi2']
    assert np.allclose(xg, xo, rtol=1e-7, atol=1e-9)


# ---------------------------------------------------------------------------
# SL/HL asymmetry (js/profile.js:608-617, :737-740, :799-826), refined
# ---------------------------------------------------------------------------
@pytest.fixture(scope='module')
def nacl_asym(nacl, oracle):
    from powder6_b200.pt_gpu import with_asymmetry
    P, M, truth = nacl
    Pa = with_asymmetry(P, 0.0, 0.0, bounds={'SL': (0.0, 0.5), 'HL': (-0.2, 0.2)})
    return Pa, oracle.PtModel(Pa, dmin=reflection_dmin(Pa)), np.append(truth, [0.2, 0.05])


def test_asymmetry_costs_and_patterns_match_oracle(nacl_asym):
    """Stretched flanks in the FP32 profile (chi^2 within 2e-6, pattern within
    2e-5 of its maximum), the doubled window and the Gauss-Legendre area
    correction in FP64, over SL 0 .. 0.4 and HL -0.1 .. 0.1."""
    P, M, x0 = nacl_asym
    xs = [x0] + [np.append(v[:-2], a) for v, a in
                 zip(start_vectors(P, x0, 4, seed=31), ([0.0, 0.0], [0.4, -0.1], [0.05, 0.1], [0.0, -0.05]))]
    with PTSession(ctx_of(P, x0, chains=len(xs))) as s:
        g, ys = s.costs(xs, with_pattern=True)
        c64 = s.model_costs(xs)
    for x, gc, gm, y in zip(xs, g, c64, ys):
        c, yo, _ = M.cost_full(P.apply(x), True)
        assert abs(gc - c) <= CHI2_RTOL * c, (gc, c)
        assert abs(gm - c) <= 1e-10 * c, (gm, c)
        assert np.max(np.abs(y - yo)) <= PATTERN_ATOL_FRAC * np.max(np.abs(yo))


def test_asymmetry_normal_equations_and_lm_match_oracle(nacl_asym):
    P, M, x0 = nacl_asym
    x = near_truth(x0)
    with PTSession(ctx_of(P, x0, chains=2)) as s:
        A, g, f = s.normal(x)
        xg, ig = s.lm(x, 30)
    Ao, go, fo = M.normal(x)
    assert abs(f - fo) <= 1e-10 * fo
    d = np.sqrt(np.diag(Ao))
    assert d[-1] > 0 and d[-2] > 0
    assert np.max(np.abs(A - Ao) / np.outer(d, d)) < 1e-7
    assert np.max(np.abs(g - go) / (d * math.sqrt(fo))) < 1e-7
    xo, io = M.lm(x, 30)
    assert ig['code'] == io['code'] and ig['accepted'] == io['accepted']
    assert abs(ig['chi2'] - io['chi2']) <= 1e-9 * io['chi2']
    assert np.allclose(xg, xo, rtol=1e-7, atol=1e-9)


# ---------------------------------------------------------------------------
# WPPF / Le Bail free intensities (js/pt_gpu.js:259-297): per evaluation, the
# non-negative heights of every reflection solved against y - background.
# The kernel's solve (coordinate descent, then an active-set polish, to a KKT
# error of 1e-5 of the largest right-hand side) and the oracle's exact
# Lawson-Hanson solve reach the same optimum; the chi^2 tolerances add, to
# the FP32 / FP64 bars above, 1e-9 of sum w y^2 for the solve's stopping rule.
# ---------------------------------------------------------------------------
FREE_SOLVE_ATOL_FRAC = 1e-9


@pytest.fixture(scope='module')
def nacl_wppf(nacl, oracle):
    import copy
    P, M, truth = nacl
    Pw = copy.copy(P)
    Pw.method = 'wppf'
    return Pw, oracle.PtModel(Pw, dmin=reflection_dmin(Pw)), truth


def test_free_intensity_costs_and_patterns_match_oracle(nacl_wppf):
    P, M, truth = nacl_wppf
    xs = [truth] + start_vectors(P, truth, 7, seed=41)
    slack = FREE_SOLVE_ATOL_FRAC * float(np.sum(P.w * P.y ** 2))
    with PTSession(ctx_of(P, truth, chains=len(xs))) as s:
        g, ys = s.costs(xs, with_pattern=True)
        c64 = s.model_costs(xs)
    for x, gc, gm, y in zip(xs, g, c64, ys):
        c, yo, _ = M.cost_full(P.apply(x), True)
        assert abs(gm - c) <= 1e-10 * c + slack, (gm, c)
        assert abs(gc - c) <= 2e-5 * c + slack, (gc, c)
        assert np.max(np.abs(y - yo)) <= PATTERN_ATOL_FRAC * np.max(np.abs(yo))


def test_free_intensity_run_reduces_chi2_and_validates(nacl_wppf):
    """Tempering with free intensities: the cell and profile move, the heights
    follow by NNLS in every proposal; the run passes the 1e-3 validation gate
    against the oracle and reaches the noise level (chi^2 below 1.2 per
    point) from a start two orders of magnitude above it."""
    P, M, truth = nacl_wppf
    x0 = start_vectors(P, truth, 1, seed=8)[0]
    c0 = M.cost(x0)
    ctx = ctx_of(P, x0, chains=32, sweeps=60, cost=M.cost)
    ctx.setup['initialCost'] = c0
    r = run(ctx)
    assert r['pt']['validationError'] < 1e-5
    assert r['pt']['bestChi2'] < 0.1 * c0
    assert abs(M.cost(r['x']) - r['pt']['bestChi2']) <= 1e-6 * r['pt']['bestChi2']


def test_free_intensity_envelope_cap_is_enforced(nacl_wppf):
    """More than 64 envelope reflections is refused at creation with an error,
    not truncated."""
    import copy
    P, _, truth = nacl_wppf
    Pb = copy.copy(P)
    Pb.values = P.values.copy()
    Pb.values[1:4] = 11.28
    Pb.lo, Pb.hi = P.lo.copy(), P.hi.copy()
    ia = P.refined.index('a')
    Pb.lo[ia], Pb.hi[ia] = 11.2, 11.4
    x = truth.copy()
    x[ia] = 11.28
    with pytest.raises(RuntimeError, match='64'):
        PTSession(ctx_of(Pb, x, chains=2))


# ---------------------------------------------------------------------------
# Sample displacement and transparency (js/pt_gpu.js:169-171, :355), refined
# ---------------------------------------------------------------------------
@pytest.fixture(scope='module')
def nacl_shift(nacl, oracle):
    from powder6_b200.pt_gpu import with_sample_shift
    P, M, truth = nacl
    Ps = with_sample_shift(P, 0.0, 0.0)
    return Ps, oracle.PtModel(Ps, dmin=reflection_dmin(Ps)), np.append(truth, [30.0, 0.002])


def test_sample_shift_costs_and_patterns_match_oracle(nacl_shift):
    """Every peak (both lines) moved by the displacement and transparency
    before the zero point: chi^2 within 2e-6 (FP32 profile) and 1e-10 (FP64
    model), pattern within 2e-5 of its maximum, over disp -80 .. 80 and
    transp -0.008 .. 0.008."""
    P, M, x0 = nacl_shift
    xs = [x0] + [np.append(v[:-2], a) for v, a in
                 zip(start_vectors(P, x0, 4, seed=33), ([0.0, 0.0], [80.0, -0.008], [-80.0, 0.008], [10.0, 0.0]))]
    with PTSession(ctx_of(P, x0, chains=len(xs))) as s:
        g, ys = s.costs(xs, with_pattern=True)
        c64 = s.model_costs(xs)
    for x, gc, gm, y in zip(xs, g, c64, ys):
        c, yo, _ = M.cost_full(P.apply(x), True)
        assert abs(gc - c) <= CHI2_RTOL * c, (gc, c)
        assert abs(gm - c) <= 1e-10 * c, (gm, c)
        assert np.max(np.abs(y - yo)) <= PATTERN_ATOL_FRAC * np.max(np.abs(yo))


def test_sample_shift_normal_equations_and_lm_match_oracle(nacl_shift):
    """The displacement and transparency columns of J'WJ (forward
    differences of 1e-2 and 1e-6) and the LM finish with their step caps (2
    and 0.01) agree with the oracle."""
    P, M, x0 = nacl_shift
    x = near_truth(x0)
    with PTSession(ctx_of(P, x0, chains=2)) as s:
        A, g, f = s.normal(x)
        xg, ig = s.lm(x, 30)
    Ao, go, fo = M.normal(x)
    assert abs(f - fo) <= 1e-10 * fo
    d = np.sqrt(np.diag(Ao))
    assert d[-1] > 0 and d[-2] > 0
    assert np.max(np.abs(A - Ao) / np.outer(d, d)) < 1e-7
    assert np.max(np.abs(g - go) / (d * math.sqrt(fo))) < 1e-7
    xo, io = M.lm(x, 30)
    assert ig['code'] == io['code'] and ig['accepted'] == io['accepted']
    assert abs(ig['chi2'] - io['chi2']) <= 1e-9 * io['chi2']
    assert np.allclose(xg, xo, rtol=1e-7, atol=1e-9)


def _philox(oracle, ctr, key):
    lib = oracle.load()
    c = np.array(ctr, dtype=np.uint32)
    k = np.array(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib.p6o_philox(c.ctypes.data, k.ctypes.data, o.ctypes.data)
    return o


def _uopen(x):
    return (float(x) + 0.5) / 4294967296.0


def _reflect(v, lo, hi):
    """The proposal's reflection into [lo, hi] (js/rietveld_core.js:2171-2241)."""
    span = hi - lo
    folded = math.fmod(math.fmod(v - lo, 2 * span) + 2 * span, 2 * span)
    return lo + (folded if folded <= span else 2 * span - folded)


def test_metropolis_and_exchange_decisions_replay_on_the_oracle(nacl, oracle):
    """Every proposal, Metropolis decision and replica exchange of four sweeps
    on eight chains, replayed on the host: the proposal from the same Philox
    words (parameter index, Gaussian step of scale x sqrt(T) reflected into
    the bounds, log u), the proposal's chi^2 from the FP64 oracle, and the
    acceptance rule (cost <= old, or log u < (old - cost) / 2T) and the
    exchange rule (la = (1/Ta - 1/Tb)(Ea - Eb)/2 >= 0, or log u < la) of
    temper.  The device's decisions are the oracle's on every move whose
    margin is not within the chi^2 tolerance, and the replayed chains end
    where the device's do."""
    P, M, truth = nacl
    chains, seed, max_t = 8, 7, 100.0
    ctx = ctx_of(P, truth, chains=chains, seed=seed, max_temp=max_t)
    scales = np.asarray(ctx.setup['scales'], dtype=np.float64)
    lo, hi = np.asarray(P.lo, dtype=np.float64), np.asarray(P.hi, dtype=np.float64)
    decided = ties = swaps_tried = 0
    with PTSession(ctx) as s:
        nv = s.plan.nv
        s.initial(start_vectors(P, truth, chains, seed=31))
        s.batch(1, True)
        s.set_trace(True)
        for k in range(4):
            x, _, costs, _ = s.exact_state()
            x, cost = x.copy(), costs[:, 0].copy()
            s.batch(1)
            x1, _, costs1, _ = s.exact_state()      # applies the exchange this sweep owes
            head, moves = s.read_trace()
            for c in range(chains):
                T = max_t ** (c / (chains - 1))
                for m in range(nv):
                    r = _philox(oracle, (k, c, m, 1), (seed, 0x2545F491))
                    j = min(nv - 1, int(_uopen(r[0]) * nv))
                    z = math.sqrt(-2.0 * math.log(_uopen(r[1]))) * math.cos(2.0 * math.pi * _uopen(r[2]))
                    xj = _reflect(x[c, j] + z * scales[j] * math.sqrt(T), lo[j], hi[j])
                    logu = math.log(_uopen(r[3]))
                    rec = moves[c, m]
                    assert int(rec[0]) == j
                    assert abs(rec[1] - xj) <= 1e-12 * max(1.0, abs(xj))
                    assert abs(rec[2] - logu) <= 1e-13
                    assert rec[3] == cost[c]
                    prop = x[c].copy()
                    prop[j] = rec[1]
                    co = M.cost(prop)
                    assert abs(rec[4] - co) <= CHI2_RTOL * co
                    acc = math.isfinite(co) and (co <= cost[c] or logu < (cost[c] - co) / (2 * T))
                    margin = min(abs(co - cost[c]), abs(logu * 2 * T - (cost[c] - co)))
                    if margin > 4 * CHI2_RTOL * co:
                        assert bool(rec[5]) == acc, (k, c, m, co, cost[c], logu)
                        decided += 1
                    else:
                        ties += 1
                    if rec[5]:
                        x[c] = prop
                        cost[c] = rec[4]
            # the exchange owed by this sweep, parity k % 2, drawn with the post-sweep counter k + 1
            par = k % 2
            new_x, new_cost = x.copy(), cost.copy()
            for c in range(chains):
                left = c if (c - par) % 2 == 0 else c - 1
                right = left + 1
                if not (left >= par and right < chains):
                    assert head[c, 0] == 0.0
                    continue
                Ta, Tb = max_t ** (left / (chains - 1)), max_t ** (right / (chains - 1))
                la = 0.5 * (1 / Ta - 1 / Tb) * (cost[left] - cost[right])
                lu = math.log(_uopen(_philox(oracle, (k + 1, left, 0x45584348, 3), (seed, 0x9E3779B9))[0]))
                swap = la >= 0 or lu < la
                assert head[c, 0] == 1.0 and abs(head[c, 2] - la) <= 1e-12 * max(1.0, abs(la))
                assert abs(head[c, 3] - lu) <= 1e-13 and bool(head[c, 1]) == swap
                swaps_tried += 1
                if swap:
                    o = right if c == left else left
                    new_x[c], new_cost[c] = x[o], cost[o]
            assert np.allclose(new_x, x1, rtol=1e-12, atol=0)
            assert np.array_equal(new_cost, costs1[:, 0])
    assert decided >= 0.9 * 4 * chains * nv and swaps_tried > 0
    print(f'PT replay: {decided} Metropolis decisions identical, {ties} within the tolerance margin, '
          f'{swaps_tried} exchange decisions identical')
