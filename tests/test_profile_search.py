"""Fixed-profile Wyckoff search, host side (no GPU): the synthetic pattern,
the product's FP64 re-score against the oracle, and the oracle's
closed-form best scale against a direct minimisation."""
import numpy as np
import pytest

from oracle import oracle as O
from powder6_b200.profile_search import profile_problem, profile_rwp, reflection_two_theta
from powder6_b200.swarm_wyckoff import reflection_intensities


@pytest.fixture(scope='module')
def pp():
    return profile_problem()


def test_closed_form_scale_is_the_minimum():
    rng = np.random.default_rng(3)
    K, N = 12, 300
    PT = np.abs(rng.normal(size=(N, K))) * (rng.random((N, K)) < 0.2)
    y = PT @ rng.lognormal(0, 1, K) * 7.0 + rng.normal(0, 0.5, N)
    w = 1.0 / np.maximum(np.abs(y), 1.0)
    w[::17] = 0.0
    I = rng.lognormal(0, 1, (5, K))
    chi, scale, syy = O.profile_fitted_chi2(I, PT, y, w)
    for r in range(5):
        Y = PT @ I[r]
        grid = scale[r] * (1 + np.linspace(-1e-3, 1e-3, 201))
        vals = [np.sum(w * (y - s * Y) ** 2) for s in grid]
        assert chi[r] <= min(vals) * (1 + 1e-12)
        assert abs(grid[int(np.argmin(vals))] / scale[r] - 1) <= 1e-5
    # a pattern no positive scale improves: chi^2 stays sum w y^2
    chi0, s0, syy0 = O.profile_fitted_chi2(I[:1], PT, -np.abs(y), w)
    assert s0[0] == 0.0 and chi0[0] == pytest.approx(syy0)


def test_product_rescore_matches_oracle(pp):
    rng = np.random.default_rng(5)
    I = rng.lognormal(0, 1.5, (6, pp.n_refl))
    chi, _, syy = O.profile_fitted_chi2(I, pp.profile_t, pp.yobs, pp.w)
    np.testing.assert_allclose(profile_rwp(pp, I), np.sqrt(chi / syy), rtol=1e-10)
    half = pp.n_points // 2
    chi_h, _, syy_h = O.profile_fitted_chi2(I, pp.profile_t, pp.yobs, pp.w, n_active=half)
    np.testing.assert_allclose(profile_rwp(pp, I, half), np.sqrt(chi_h / syy_h), rtol=1e-10)


def test_intensities_match_oracle(pp):
    prob = pp.problem
    ms = prob.tables.max_sites
    rng = np.random.default_rng(9)
    for x in (prob.true_coords, rng.random(ms * 3)):
        xp = np.zeros(ms * 3)
        for si, s in enumerate(prob.assignments[0].sites):
            xp[si * 3:si * 3 + 3] = np.array(s.w.project(*x[si * 3:si * 3 + 3])) % 1.0
        a = reflection_intensities(prob, xp, 0)
        b = O.wy_reflection_intensities(prob, 0, xp)
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-9 * float(np.max(b)))


def test_pattern_shape(pp):
    # reflections in 2-theta order, each column a peak inside the pattern
    assert np.all(np.diff(pp.tth_refl) >= 0)
    np.testing.assert_allclose(pp.tth_refl, reflection_two_theta(pp.problem, 1.5406))
    assert pp.profile_t.shape == (pp.n_points, pp.n_refl)
    assert np.all(pp.profile_t >= 0) and np.all(pp.profile_t.max(axis=0) > 0)
    peak_at = pp.tth[np.argmax(pp.profile_t, axis=0)]
    assert np.max(np.abs(peak_at - pp.tth_refl)) <= 0.011
    # the true structure sits at the noise floor; random structures far above it
    rng = np.random.default_rng(2)
    prob = pp.problem
    ms = prob.tables.max_sites
    rnd = []
    for _ in range(8):
        x = np.zeros(ms * 3)
        for si, s in enumerate(prob.assignments[0].sites):
            x[si * 3:si * 3 + 3] = np.array(s.w.project(*rng.random(3))) % 1.0
        rnd.append(reflection_intensities(prob, x, 0))
    r = profile_rwp(pp, np.array(rnd))
    assert 0.0 < pp.rwp_true < 0.2
    assert np.min(r) > 2.0 * pp.rwp_true


def test_gram_form_equals_the_pattern_chi2(pp):
    from powder6_b200.profile_search import gram_operands
    v, band, bw, syy = gram_operands(pp)
    assert band.shape == (bw + 1, pp.n_refl) and 0 < bw < pp.n_refl
    rng = np.random.default_rng(11)
    I = rng.lognormal(0, 1.5, (5, pp.n_refl))
    K = pp.n_refl
    G = np.zeros((K, K))
    for d in range(bw + 1):
        G[np.arange(K - d), np.arange(d, K)] = band[d, :K - d]
        G[np.arange(d, K), np.arange(K - d)] = band[d, :K - d]
    a = I @ v
    b = np.einsum('rk,kl,rl->r', I, G, I)
    chi = np.where((a > 0) & (b > 0), syy - a * a / b, syy)
    chi64, _, syy64 = O.profile_fitted_chi2(I, pp.profile_t, pp.yobs, pp.w)
    assert syy == pytest.approx(syy64, rel=1e-12)
    np.testing.assert_allclose(chi, chi64, rtol=1e-10)


def test_sparse_pattern_matches_the_dense_one(pp):
    from powder6_b200.profile_search import gram_operands, pattern_gram
    pg = pattern_gram(pp.problem, seed=1)
    v, band, bw, syy = gram_operands(pp)
    assert pg.n_points == pp.n_points and pg.bw == bw
    np.testing.assert_allclose(pg.v, v, rtol=1e-5, atol=1e-6 * np.max(np.abs(v)))
    np.testing.assert_allclose(pg.band, band, rtol=1e-5, atol=1e-6 * np.max(band))
    assert pg.syy == pytest.approx(syy, rel=1e-9)
    assert pg.rwp_true == pytest.approx(pp.rwp_true, rel=1e-5)
