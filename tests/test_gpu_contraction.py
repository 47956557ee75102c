"""Split-BF16 tensor-core contraction and the FP32 CUDA-core contraction
against the FP64 oracle.

Bars: the split-BF16 product drops the I_lo P_lo term (~2^-16 relative) and
rounds the low parts to bf16, so each element of Y is within 4e-5 of the
sum of |I||P| over its band; the FP32 product within 4e-6.  chi^2 per
replica: split-BF16 within 2e-5 relative of FP64, FP32 within 2e-6 (both
stated in the tests below).  The three-part split (six products, every
operand to 2^-27) within 6e-6 of the bound per element and 6e-6 relative in
chi^2: what is left is the tensor core's FP32 accumulation (measured 3.6e-6
and 3.7e-6, where the FP32 CUDA-core product gives 1.3e-6 and 3.4e-7)."""
import numpy as np
import pytest

from powder6_b200.contraction import FP32, SPLIT3_BF16, SPLIT_BF16, ContractionSession, banded_problem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def small():
    # 300 replicas (3 row tiles, the last partial), 700 reflections (11 K-blocks,
    # the last partial), 3000 points (12 column tiles, the last partial)
    return banded_problem(n_refl=700, n_points=3000, n_replicas=300, seed=11)


def bound(p):
    return np.abs(p.intensities.astype(np.float64)) @ np.abs(p.profile_t.astype(np.float64)).T


@pytest.mark.parametrize('method,tol_y,tol_chi', [(SPLIT_BF16, 4e-5, 5e-5), (FP32, 2e-5, 1e-5),
                                             (SPLIT3_BF16, 6e-6, 6e-6)])
def test_contraction_matches_fp64(oracle, small, method, tol_y, tol_chi):
    p = small
    Y64, chi64 = oracle.contract_fp64(p.intensities, p.profile_t, p.yobs, p.w)
    with ContractionSession(p) as s:
        chi, Y = s.run(p.intensities, method, pattern=True)
    B = bound(p)
    ey = float(np.max(np.abs(Y - Y64) / np.maximum(B, 1e-30)))
    ec = float(np.max(np.abs(chi - chi64) / chi64))
    print(f'method {method}: max |dY| / sum |I||P| {ey:.2e}, max rel d chi^2 {ec:.2e}')
    assert ey <= tol_y
    assert ec <= tol_chi


def test_two_calls_in_a_row_and_fewer_replicas(oracle, small):
    p = small
    with ContractionSession(p) as s:
        c1 = s.run(p.intensities, SPLIT_BF16)
        c2 = s.run(p.intensities[:77], SPLIT_BF16)
        c3 = s.run_host(p.intensities, SPLIT_BF16)
    assert np.array_equal(c1[:77], c2) and np.array_equal(c1, c3)
    _, chi64 = oracle.contract_fp64(p.intensities[:77], p.profile_t, p.yobs, p.w)
    assert np.max(np.abs(c2 - chi64) / chi64) <= 5e-5


def test_empty_band_tiles_give_the_observed_chi2(oracle):
    """Points no reflection reaches contribute w yobs^2 (y_calc = 0 there)."""
    p = banded_problem(n_refl=64, n_points=2048, n_replicas=128, seed=5, tth0=5.0, step=0.05)
    p.profile_t[1024:, :] = 0.0            # no reflection reaches the upper half
    _, chi64 = oracle.contract_fp64(p.intensities, p.profile_t, p.yobs, p.w)
    with ContractionSession(p) as s:
        q = s.query()
        chi = s.run(p.intensities, SPLIT_BF16)
    assert q['n_tiles'] == 8
    assert np.max(np.abs(chi - chi64) / chi64) <= 5e-5


def test_full_size_sample_rows(oracle):
    """16384 x 3000 x 12000 workload: 64 sampled replicas against FP64."""
    p = banded_problem(seed=1)
    rows = np.linspace(0, len(p.intensities) - 1, 64).astype(int)
    with ContractionSession(p) as s:
        chi_s = s.run(p.intensities, SPLIT_BF16)
        chi_f = s.run(p.intensities, FP32)
        chi_3 = s.run(p.intensities, SPLIT3_BF16)
    _, chi64 = oracle.contract_fp64(p.intensities[rows], p.profile_t, p.yobs, p.w)
    assert np.max(np.abs(chi_s[rows] - chi64) / chi64) <= 5e-5
    assert np.max(np.abs(chi_f[rows] - chi64) / chi64) <= 1e-5
    e3 = float(np.max(np.abs(chi_3[rows] - chi64) / chi64))
    print(f'full size, three-part split: max rel d chi^2 {e3:.2e}')
    assert e3 <= 6e-6
