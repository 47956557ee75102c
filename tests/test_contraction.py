"""The fixed-profile contraction workload and its FP64 oracle (CPU)."""
import numpy as np

from powder6_b200.contraction import banded_problem, pseudo_voigt


def test_banded_problem_shapes_and_band():
    p = banded_problem(n_refl=200, n_points=1500, n_replicas=32, seed=3)
    assert p.profile_t.shape == (1500, 200) and p.intensities.shape == (32, 200)
    assert np.all(np.diff(p.centres) >= 0)
    assert np.all((p.fwhm >= 0.05) & (p.fwhm <= 0.3))
    # every column is a unit-height peak at its centre, zero beyond +/- 20 FWHM
    for r in (0, 57, 199):
        col = p.profile_t[:, r]
        nz = np.nonzero(col)[0]
        assert np.all(np.abs(p.tth[nz] - p.centres[r]) <= 20 * p.fwhm[r] + 1e-9)
        j = int(np.argmin(np.abs(p.tth - p.centres[r])))
        assert abs(col[j] - pseudo_voigt(p.tth[j] - p.centres[r], p.fwhm[r], p.eta[r])) < 1e-6
    assert np.all(p.w > 0) and np.all(np.isfinite(p.yobs))


def test_fp64_oracle_is_the_weighted_residual(oracle):
    p = banded_problem(n_refl=50, n_points=400, n_replicas=4, seed=4)
    Y, chi = oracle.contract_fp64(p.intensities, p.profile_t, p.yobs, p.w)
    j = 123
    y = sum(float(p.intensities[1, k]) * float(p.profile_t[j, k]) for k in range(50))
    assert abs(Y[1, j] - y) <= 1e-12 * max(1.0, abs(y))
    r = p.yobs.astype(np.float64) - Y[2]
    assert abs(chi[2] - float(np.sum(p.w.astype(np.float64) * r * r))) <= 1e-9 * chi[2]
