"""Fixed-profile Wyckoff search on the GPU against the FP64 oracle.

Bars (relative error of chi^2 at the best scale, per replica, against the
oracle's FP64 closed form): split-BF16 on the tensor cores 3e-5, the
three-part split 1e-6, the FP32 CUDA-core products (banded and dense) 5e-7;
the fitted scale, which chi^2 does not depend on to first order, to ten
times those.  Near the true structure, where chi^2 is a
small difference of large sums, the same bars hold (the structures at and
around the truth).  In the search, a replica's 1 - Rwp is kept in FP32, so
Rwp is compared to Rwp * tol / 2 + 2e-7 absolute; the Gram form inside the
fused search (exact FP64, no pattern formed) to the same FP32 rounding.  The
acceptance of one generation is replayed on the host from the recorded
proposal, penalty and uniform: the same decisions, and the accepted
proposals become the current structures."""
import numpy as np
import pytest

from powder6_b200.contraction import ContractionSession, banded_problem
from powder6_b200.profile_search import (FP32, FP32_DENSE, GRAM_FP64, SPLIT3_BF16, SPLIT_BF16, ProfileSearch,
                                         profile_problem, run_profile_search)
from powder6_b200.swarm_wyckoff import schedule

pytestmark = pytest.mark.gpu

TOL = {SPLIT_BF16: 3e-5, SPLIT3_BF16: 1e-6, FP32: 5e-7, FP32_DENSE: 5e-7, GRAM_FP64: 1e-9}


@pytest.fixture(scope='module')
def small():
    return banded_problem(n_refl=700, n_points=3000, n_replicas=300, seed=11)


@pytest.fixture(scope='module')
def pp():
    return profile_problem()


@pytest.mark.parametrize('method', [SPLIT_BF16, SPLIT3_BF16, FP32, FP32_DENSE])
def test_fitted_chi2_matches_fp64(oracle, small, method):
    p = small
    with ContractionSession(p) as s:
        s.set_fitted(True)
        chi = s.run(p.intensities, method)
        scale = s.read_scale()
    chi64, s64, _ = oracle.profile_fitted_chi2(p.intensities, p.profile_t, p.yobs, p.w)
    ec = float(np.max(np.abs(chi - chi64) / chi64))
    es = float(np.max(np.abs(scale - s64) / s64))
    print(f'method {method}: chi^2 {ec:.2e}, scale {es:.2e}')
    assert ec <= TOL[method] and es <= 10 * TOL[method]


@pytest.mark.parametrize('method', [SPLIT_BF16, SPLIT3_BF16, FP32, FP32_DENSE])
def test_fitted_chi2_near_the_truth(oracle, pp, method):
    from powder6_b200.swarm_wyckoff import reflection_intensities
    from powder6_b200.profile_search import _ContractionInput
    I0 = reflection_intensities(pp.problem, pp.problem.true_coords, 0)
    rng = np.random.default_rng(4)
    eps = np.repeat([0.0, 1e-3, 1e-2, 3e-2, 0.1, 0.3], 32)
    I = (I0[None, :] * np.exp(eps[:, None] * rng.normal(size=(len(eps), len(I0))))).astype(np.float32)
    with ContractionSession(_ContractionInput(pp), max_replicas=len(I)) as s:
        s.set_fitted(True)
        chi = s.run(I, method)
    chi64, _, syy = oracle.profile_fitted_chi2(I, pp.profile_t, pp.yobs, pp.w)
    ec = np.abs(chi - chi64) / chi64
    print(f'method {method}: near the truth chi^2 {ec.max():.2e} (Rwp {np.sqrt(chi64.min() / syy):.4f}..'
          f'{np.sqrt(chi64.max() / syy):.4f})')
    assert ec.max() <= TOL[method]


def oracle_rwp(oracle, pp, fixed, assign_of):
    prob = pp.problem
    cpp = prob.tables.max_sites * 3
    x = fixed.astype(np.float64).reshape(-1, cpp) / 2.0 ** 32
    I = np.array([oracle.wy_reflection_intensities(prob, int(a), x[i]) for i, a in enumerate(assign_of)])
    chi, _, syy = oracle.profile_fitted_chi2(I, pp.profile_t, pp.yobs, pp.w)
    return np.sqrt(chi / syy)


@pytest.mark.parametrize('method', [SPLIT_BF16, FP32_DENSE, GRAM_FP64])
def test_first_evaluation_matches_oracle(oracle, pp, method):
    with ProfileSearch(pp, 256, run_key=7) as ps:
        ps.start(200, seed=3, method=method)
        ps.synchronize()
        _, _, st = ps.wy.read_state()
        cur, best = ps.wy.read_positions_fixed()
        assign_of = ps.assign_of.copy()
    r = oracle_rwp(oracle, pp, cur, assign_of)
    err = np.abs((1.0 - st['cc'].astype(np.float64)) - r)
    print(f'method {method}: max |Rwp - Rwp64| {err.max():.2e} (Rwp {r.min():.3f}..{r.max():.3f})')
    assert np.all(err <= r * TOL[method] / 2 + 2e-7)
    if method != GRAM_FP64:   # the fused search's first evaluation leaves the bests to the first move
        np.testing.assert_array_equal(best, cur)
        np.testing.assert_array_equal(st['best_cc'], st['cc'])


def test_generation_replays_on_oracle(oracle, pp):
    n, G = 256, 100
    _, pen_sched = schedule(G, pp.problem.refl.n_groups)
    with ProfileSearch(pp, n, run_key=11) as ps:
        ps.start(G, seed=5, method=FP32_DENSE)
        ps.run(0, 3, FP32_DENSE, swap_every=0)
        ps.synchronize()
        cur0, _ = ps.wy.read_positions_fixed()
        _, _, st0 = ps.wy.read_state()
        ps.run(3, 1, FP32_DENSE, swap_every=0)
        ps.synchronize()
        props, rec = ps.wy.read_trace()
        cur1, best1 = ps.wy.read_positions_fixed()
        _, _, st1 = ps.wy.read_state()
        assign_of = ps.assign_of.copy()
    cpp = pp.problem.tables.max_sites * 3
    # every proposal's 1 - Rwp is the oracle's
    r = oracle_rwp(oracle, pp, props, assign_of)
    assert np.all(np.abs((1.0 - rec[:, 1].astype(np.float64)) - r) <= r * TOL[FP32_DENSE] / 2 + 2e-7)
    # the Metropolis decisions from the recorded energies and uniforms
    ps3 = np.float32(pen_sched[3])
    f_old = (st0['cc'] - st0['pen'] * ps3).astype(np.float32)
    np.testing.assert_allclose(rec[:, 5], f_old, rtol=0, atol=1e-6)
    f_old = rec[:, 5]
    f_new = rec[:, 0]
    ratio = np.exp(np.minimum((f_new - f_old) / np.maximum(st0['temp'], np.float32(1e-9)), 0.0).astype(np.float64))
    want = (f_new >= f_old) | (rec[:, 3] < ratio)
    clear = np.abs(rec[:, 3] - ratio) > 1e-6
    acc = rec[:, 4] > 0.5
    np.testing.assert_array_equal(acc[clear], want[clear])
    assert 0 < acc.sum() < n
    np.testing.assert_array_equal(st1['accepted'] - st0['accepted'], acc.astype(np.uint32))
    for i in range(n):
        sl = slice(i * cpp, (i + 1) * cpp)
        np.testing.assert_array_equal(cur1[sl], props[sl] if acc[i] else cur0[sl])
    # the best of each replica, judged by fitness at this generation's penalty weight, never gets worse
    b0 = st0['best_cc'] - st0['best_pen'] * ps3
    b1 = st1['best_cc'] - st1['best_pen'] * ps3
    assert np.all(b1 >= b0 - 1e-6)


@pytest.mark.parametrize('method', [SPLIT_BF16, FP32_DENSE, GRAM_FP64])
def test_search_improves_and_rescore_agrees(pp, method):
    res = run_profile_search(pp, num_particles=1024, generations=400, seed=2, method=method, chunk=100)
    print(f'{res.method}: best Rwp {res.best_rwp:.4f} (true {pp.rwp_true:.4f}), {res.device_ms:.1f} ms, '
          f'accept {res.accept_rate:.2f}, check {res.cpu_check}')
    assert res.best_rwp < 0.5
    assert res.cpu_check['delta'] <= res.best_rwp * TOL[method] + 1e-6


def test_gram_form_in_the_fp32_cosine_mode(oracle, pp):
    # cos mode 1 (FMA polynomial): FP32 intensities (|F|^2 within 5e-6 relative of the largest), FP64 sums
    with ProfileSearch(pp, 256, run_key=9, cos_mode=1) as ps:
        ps.start(200, seed=4, method=GRAM_FP64)
        ps.synchronize()
        _, _, st = ps.wy.read_state()
        cur, _ = ps.wy.read_positions_fixed()
        assign_of = ps.assign_of.copy()
    r = oracle_rwp(oracle, pp, cur, assign_of)
    err = np.abs((1.0 - st['cc'].astype(np.float64)) - r)
    print(f'cos mode 1, Gram form: max |Rwp - Rwp64| {err.max():.2e}')
    assert np.all(err <= 2e-5 * r + 2e-7)


def test_profile_run_refuses_mismatched_sessions(pp):
    from powder6_b200._lib import P6Error, check
    from powder6_b200.profile_search import _ContractionInput
    with ProfileSearch(pp, 128, run_key=2) as ps:
        ps.prepare(50, seed=2)
        lib = ps.lib
        # a contraction over other reflections
        other = banded_problem(n_refl=pp.n_refl + 8, n_points=1000, n_replicas=128, seed=3)
        with ContractionSession(other, max_replicas=128) as ct:
            with pytest.raises(P6Error) as e:
                check(lib.p6_wy_profile_run(ps.wy.h, ct.h, SPLIT_BF16, 0, 1, 10, 1, 0))
            assert e.value.status == 'INVALID_ARG'
        # a contraction holding fewer replicas than the search
        with ContractionSession(_ContractionInput(pp), max_replicas=64) as ct:
            with pytest.raises(P6Error) as e:
                check(lib.p6_wy_profile_run(ps.wy.h, ct.h, SPLIT_BF16, 0, 1, 10, 1, 0))
            assert e.value.status == 'CAPACITY'
        # generations outside the schedule, an unknown method
        with pytest.raises(P6Error):
            ps.run(40, 20, SPLIT_BF16)
        with pytest.raises(P6Error):
            check(lib.p6_wy_profile_run(ps.wy.h, ps.ct.h, 9, 0, 1, 10, 0, 0))
        # Gram operands without weighted counts
        v = np.zeros(pp.n_refl)
        with pytest.raises(P6Error):
            check(lib.p6_wy_set_profile(ps.wy.h, v.ctypes.data, v.ctypes.data, 0, 0.0))
        # the session still runs after the refusals
        ps.run(0, 5, SPLIT_BF16, init=True)
        ps.synchronize()
