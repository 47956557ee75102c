"""Wyckoff-constrained coordinate refinement (js/coord_refine.js:266-627):
the FP64 restatement's analytic Jacobian against finite differences, and
its refinement from a perturbed structure back to the true one's residual
with every site kept on its Wyckoff subspace."""
import numpy as np

from oracle import oracle as O
from powder6_b200.workloads import wyckoff_problem


def test_constrained_jacobian_matches_finite_differences():
    P = wyckoff_problem(seed=1)
    ms = P.tables.max_sites
    x0 = P.true_coords.copy()
    _, J = O.wy_refine_intensities(P, 0, x0, jac=True)
    _, projs, *_ = O._refine_tables(P, 0)
    worst, checked = 0.0, 0
    for si, (Pm, _) in enumerate(projs):
        for c in range(3):
            if abs(Pm[c, c]) < 0.5:
                assert np.all(J[:, 3 * si + c] == 0)          # a fixed direction has no derivative
                continue
            e = np.zeros(ms * 3)
            e[3 * si + c] = 1e-6
            ip, _ = O.wy_refine_intensities(P, 0, x0 + e)
            im, _ = O.wy_refine_intensities(P, 0, x0 - e)
            worst = max(worst, float(np.max(np.abs((ip - im) / 2e-6 - J[:, 3 * si + c])) / np.max(np.abs(J))))
            checked += 1
    assert checked == 11                                      # 4 x (x, z) of 4c + (x, y, z) of 8d
    assert worst < 1e-7


def test_refinement_returns_to_the_true_residual_on_the_subspaces():
    P = wyckoff_problem(seed=1)
    rng = np.random.default_rng(3)
    x_true = P.true_coords.copy()
    x_r, r0, r1, chi, steps, conv = O.wy_refine(P, 0, x_true + rng.uniform(-0.003, 0.003, x_true.shape))
    _, rt, _, _, _, _ = O.wy_refine(P, 0, x_true, max_iter=0)
    assert conv and steps > 5
    assert r0 > 5 * r1
    assert r1 <= rt                                           # at least as good as the (noisy) truth
    y = x_r.reshape(-1, 3)
    for si, st in enumerate(P.assignments[0].sites):
        if st.w.triplet == 'x,1/4,z':
            assert abs(y[si, 1] - 0.25) < 1e-12
    d = (y - x_true.reshape(-1, 3) + 0.5) % 1.0 - 0.5
    assert np.max(np.abs(d)) < 5e-3
