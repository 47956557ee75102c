"""Charge flipping on the B200 against the FP64 restatement of the cycle.

The device computes in FP32 as the reference's kernels do
(charge_flipping.wgsl), with the flip threshold's moments, the cluster sums
and the R factor in FP64.  The flip is a discontinuity: a point whose density
lies within FP32 rounding of the threshold may flip either way, so a cycle is
compared only when the oracle's density keeps every point at least 1e-5
sigma from the threshold, and the device error is well inside that band.
Tolerances: R within 1e-5, |F| within 2e-5 of max |F|, F within that plus
the amplitude constraint's conditioning (below)."""
import numpy as np
import pytest

from powder6_b200.charge_flipping import (CFSession, build_reflection_model, classify_weak_orbits,
                                          model_initial_grid, run_charge_flipping, synthetic_job)

pytestmark = pytest.mark.gpu

N = 32


@pytest.fixture(scope='module')
def model():
    job = synthetic_job()
    m = build_reflection_model(job, N)
    return job, m, classify_weak_orbits(m, 0.15, 'cluster')['flags']


def settings(weak):
    return [{'threshold': 1.1, 'symLambda': 0.0, 'seed': 13, 'weak': None},
            {'threshold': 1.0, 'symLambda': 0.5, 'seed': 13, 'weak': weak},
            {'threshold': 1.2, 'symLambda': 1.0, 'seed': 13, 'weak': None},
            {'threshold': 1.1, 'symLambda': 0.75, 'seed': 13, 'weak': weak}]


def test_every_cycle_matches_oracle(model):
    """P1 flipping, damped and strict symmetrisation, weak-orbit quarter-turns:
    four trials of one batch, six cycles.  Flipping amplifies any difference
    between two runs by an order of magnitude a cycle (a start that obeys the
    space group is unstable to antisymmetric perturbations without
    symmetrisation), so each cycle is checked from the device's own previous
    grid: the oracle runs one cycle from it and the device's next grid and R
    must agree: R within 1e-5, every |F| within 2e-5 of max |F|, and every F
    within that plus the phase error that a transform error of 1e-6 of its
    largest value causes when the amplitude constraint rescales a member from
    its post-transform magnitude (ill-conditioned for small magnitudes: a
    perturbation of 1e-6 moves some members' phases by radians, in the FP64
    oracle as well).  A cycle whose input puts a point within 1e-5 sigma of
    the threshold is not compared (at most six of the 24 may be skipped).  The best grid is the device's grid of the
    cycle with the lowest R, bit for bit."""
    from oracle.oracle_cf import CfState
    _, m, weak = model
    trials = settings(weak)
    start = model_initial_grid(m, N, 13)
    compared = 0
    with CFSession(m, trials) as s:
        s.set_grid(start)
        prev = [start.astype(np.float64)] * len(trials)
        grids = [[] for _ in trials]
        hist = [[] for _ in trials]
        for c in range(6):
            r = s.run(1)[:, 0]
            for t, tr in enumerate(trials):
                g = s.read(t, 'current')
                st = CfState(m, prev[t], tr['threshold'], tr['symLambda'], tr['seed'], tr['weak'])
                ro = st.cycle()
                if st.ambiguous(1e-5) == 0:
                    gc = g[0::2].astype(np.float64) + 1j * g[1::2]
                    base = 2e-5 * np.max(np.abs(st.F))
                    # magnitudes (targets from cluster sums) are well conditioned everywhere
                    dm = np.abs(np.abs(gc) - np.abs(st.F))
                    assert np.max(dm) <= base, (c, t, np.max(dm))
                    # phases: within what the transform's rounding allows after the rescaling
                    d = np.abs(gc - st.F)
                    assert np.all(d <= st.tolerance(base, 1e-6)), (c, t, np.max(d / st.tolerance(base, 1e-6)))
                    assert abs(r[t] - ro) <= 1e-5, (c, t, r[t], ro)
                    compared += 1
                prev[t] = g.astype(np.float64)
                grids[t].append(g)
                hist[t].append(r[t])
        best_r = s.best_r()
        for t in range(len(trials)):
            k = int(np.argmin(hist[t]))
            assert best_r[t] == hist[t][k]
            assert np.array_equal(s.read(t, 'best'), grids[t][k])
    assert compared >= 18


def test_trials_are_independent_and_deterministic(model):
    """A trial computes the same bits alone and inside a batch of four, and a
    repeated run reproduces them."""
    _, m, weak = model
    trials = settings(weak)
    start = model_initial_grid(m, N, 3)
    with CFSession(m, trials) as s:
        s.set_grid(start)
        h4 = s.run(5)
        g4 = s.read(1, 'current')
    with CFSession(m, [trials[1]]) as s:
        s.set_grid(start)
        h1 = s.run(5)
        g1 = s.read(0, 'current')
        s.set_grid(start)
        h1b = s.run(5)
        g1b = s.read(0, 'current')
    assert np.array_equal(h4[1], h1[0]) and np.array_equal(g4, g1)
    assert np.array_equal(h1, h1b) and np.array_equal(g1, g1b)


def test_density_of_the_best_grid(model):
    """The map read back is the real part of the inverse transform of the
    best grid, 1/n^3 included (within 1e-5 of its maximum)."""
    _, m, weak = model
    with CFSession(m, settings(weak)[:1]) as s:
        s.set_grid(model_initial_grid(m, N, 5))
        s.run(3)
        b = s.read(0, 'best').astype(np.float64)
        rho = s.read(0, 'map')
    ref = np.fft.ifftn((b[0::2] + 1j * b[1::2]).reshape(N, N, N)).ravel().real
    assert np.max(np.abs(rho - ref)) <= 1e-5 * np.max(np.abs(ref))


def test_run_converges_on_the_synthetic_structure():
    """run_charge_flipping: P1 flipping on the exact intensities of the
    synthetic P2_1/c structure reaches R < 0.1 in 200 cycles (the oracle
    reaches 0.043 in 150 from the same start), in a batch with the adaptive
    plan's other settings; the best trial's R is its history's minimum."""
    job = synthetic_job(overlap_tol=0.0, maxIterations=200, seed=543, symLambda=0.0, weakFraction=0.0)
    out = run_charge_flipping(job, trials=[{}, {'threshold': 1.1, 'symLambda': 0.5, 'weakFraction': 0.15},
                                           {'threshold': 1.2, 'symLambda': 0.5, 'weakFraction': 0.2}])
    assert out['trials'][0]['bestR'] < 0.1
    assert out['bestR'] == min(t['bestR'] for t in out['trials'])
    assert abs(out['bestR'] - float(np.nanmin(out['rHistory']))) <= 1e-7
    assert out['map'].shape == (N ** 3,) and np.isfinite(out['map']).all()


def test_create_rejects_inconsistent_models(model):
    """A grid edge that is not a power of two from 8 to 128, and a grid point
    claimed by two members, are refused at creation."""
    from powder6_b200._lib import P6Error
    _, m, _ = model
    bad = dict(m, N=24)
    with pytest.raises(P6Error):
        CFSession(bad, [{'threshold': 1.1}])
    dup = dict(m)
    dup['orbit_idx'] = m['orbit_idx'].copy()
    dup['orbit_idx'][1] = dup['orbit_idx'][0]
    with pytest.raises(P6Error, match='claimed twice'):
        CFSession(dup, [{'threshold': 1.1}])
