"""Charge flipping: the reflection model, random starts and weak-orbit
classification of the host layer against the reference's own tests
(tests/cf-physics.test.cjs:5-35), the systematic absences against their
definition, and the FP64 cycle restatement (the oracle) against direct
arithmetic and its convergence on a known structure."""
import math

import numpy as np
import pytest

from powder6_b200.charge_flipping import (CONJ_BIT, IDX_MASK, build_reflection_model, cf_plan, classify_weak_orbits,
                                          find_systematic_absences, model_initial_grid, normalize_symops,
                                          synthetic_job)

IDENTITY = {'r': [1, 0, 0, 0, 1, 0, 0, 0, 1], 't': [0, 0, 0]}


def inversion(t):
    return {'r': [-1, 0, 0, 0, -1, 0, 0, 0, -1], 't': list(t)}


def physics_job(symops):
    """The job of tests/cf-physics.test.cjs:7: a 16^3 grid, eight reflections
    (h, k, l) = (i % 3 + 1, i // 3, 1), intensities 10 (i + 1), 2-theta 10 + i."""
    return {'gridSize': 16, 'maxIterations': 1, 'thresholdSigma': 1.1, 'seed': 543, 'symops': symops,
            'symLambda': .5, 'weakFraction': .25, 'weakGrouping': 'individual', 'overlapTolTth': .001,
            'applyLP': False,
            'hklList': [{'h_orig': i % 3 + 1, 'k_orig': i // 3, 'l_orig': 1, 'intensity': (i + 1) * 10,
                         'tth': 10 + i} for i in range(8)]}


def density(init, N):
    F = (init[0::2].astype(np.float64) + 1j * init[1::2]).reshape(N, N, N)
    return np.fft.ifftn(F)


@pytest.mark.parametrize('t', [(0, 0, 0), (.5, .25, 0)])
def test_centric_starts_have_the_measured_amplitudes_and_a_real_map(t):
    """tests/cf-physics.test.cjs:8-17: every member starts at |F|^2 =
    target / count (1e-6), and the start's density is real (imaginary energy
    below 1e-12 of the real), with the inversion centre at the origin or
    translated."""
    j = physics_job([IDENTITY, inversion(t)])
    m = build_reflection_model(j, 16)
    init = model_initial_grid(m, 16, j['seed'])
    for g in range(m['n_orbits']):
        expected = m['orbit_target_i'][g] / m['orbit_count'][g]
        for p in range(m['orbit_start'][g], m['orbit_start'][g] + m['orbit_count'][g]):
            i = int(m['orbit_idx'][p]) & IDX_MASK
            assert abs(init[2 * i] ** 2 + init[2 * i + 1] ** 2 - expected) < 1e-6 * expected
    rho = density(init, 16)
    assert np.sum(rho.imag ** 2) < 1e-12 * np.sum(rho.real ** 2)


@pytest.mark.parametrize('number', [1, 2, 12, 14, 15, 62, 166, 176, 221, 225])
def test_space_groups_initialise_a_real_density(number):
    """tests/cf-physics.test.cjs:18-30 over the groups this package carries:
    reflections 0 <= h < 3, |k|, |l| <= 2 on an 8^3 grid build a model with no
    error and a start whose density is real."""
    from powder6_b200.symmetry import space_group
    hkl = []
    for h in range(3):
        for k in range(-2, 3):
            for l in range(-2, 3):
                if h or k or l:
                    hkl.append({'h_orig': h, 'k_orig': k, 'l_orig': l, 'intensity': 100 + 2 * h + k + l,
                                'tth': len(hkl) + 1})
    m = build_reflection_model({'symops': space_group(number).op_dicts(), 'applyLP': False,
                                'overlapTolTth': 1e-8, 'hklList': hkl}, 8)
    assert 'error' not in m
    rho = density(model_initial_grid(m, 8, 43), 8)
    assert np.sum(rho.imag ** 2) < 1e-12 * np.sum(rho.real ** 2)


def test_model_invariants():
    """Members are unique grid points (none absent, none F(000)); the
    members of an orbit are the Laue orbit with Friedel mates (powder
    multiplicity); the cluster intensity is the sum of its orbits' shares; the
    absent list is the tail of orbitIdx."""
    j = synthetic_job()
    m = build_reflection_model(j, 32)
    nm = m['n_members']
    idx = m['orbit_idx'][:nm] & IDX_MASK
    absent = m['orbit_idx'][nm:]
    assert len(np.unique(idx)) == nm and 0 not in idx
    assert not set(idx.tolist()) & set(absent.tolist())
    # P2_1/c: Laue 2/m orbits of 2 or 4 members, the powder multiplicities
    assert set(m['orbit_count'].tolist()) <= {2, 4}
    absent_set = set(absent.tolist())
    allowed = [q for q in j['hklList']
               if (q['h_orig'] % 32) + (q['k_orig'] % 32) * 32 + (q['l_orig'] % 32) * 1024 not in absent_set]
    assert nm == sum(q['multiplicity'] for q in allowed)
    for c in range(m['n_clusters']):
        s, n = m['cluster_orbit_start'][c], m['cluster_n_orbits'][c]
        assert m['cluster_obs_i'][c] >= np.sum(m['orbit_target_i'][s:s + n]) * (1 - 1e-6)


def test_systematic_absences_p21c():
    """P2_1/c (b unique): h0l with l odd and 0k0 with k odd are extinct, and
    nothing else (on a 16^3 grid)."""
    from powder6_b200.symmetry import space_group
    N = 16
    ab = set(find_systematic_absences(N, normalize_symops(space_group(14).op_dicts())).tolist())
    expect = set()
    half = N // 2
    for ml in range(N):
        for mk in range(N):
            for mh in range(N):
                h, k, l = (v - N if v > half else v for v in (mh, mk, ml))
                if (k == 0 and l % 2) or (h == 0 and l == 0 and k % 2):
                    expect.add(mh + mk * N + ml * N * N)
    assert ab == expect


def test_systematic_absences_centring_without_operators():
    """An F lattice given only by its letter: h, k, l of mixed parity."""
    N = 8
    ab = set(find_systematic_absences(N, None, 'F').tolist())
    half = N // 2
    for ml in range(N):
        for mk in range(N):
            for mh in range(N):
                h, k, l = (v - N if v > half else v for v in (mh, mk, ml))
                mixed = len({h % 2, k % 2, l % 2}) > 1
                assert ((mh + mk * N + ml * N * N) in ab) == mixed


def test_weak_classification_and_plan():
    """The weakest fraction of units is flagged (individual orbits or whole
    clusters), and the adaptive plan cycles its three settings over the
    starts (js/cf_adaptive.js:43-51)."""
    j = physics_job([IDENTITY, inversion((0, 0, 0))])
    m = build_reflection_model(j, 16)
    w = classify_weak_orbits(m, .25, 'individual')
    assert w['weak_orbits'] == 2 and w['flags'].sum() == 2
    per = m['orbit_target_i'] / m['orbit_count']
    assert set(np.nonzero(w['flags'])[0]) == set(np.argsort(per, kind='stable')[:2])
    p = cf_plan(9)
    assert [t['threshold'] for t in p['trials'][:3]] == [1.0, 1.1, 1.2]
    assert [s['starts'] for s in p['settings']] == [3, 3, 3]
    with pytest.raises(ValueError):
        cf_plan(4)


def test_oracle_cycle_steps():
    """One oracle cycle against direct arithmetic: the flip threshold is
    delta_sigma times the population sigma of Re rho; after the cycle every
    non-weak orbit has equal member amplitudes sqrt(target / count), the
    absent reflections and F(000) are zero, and R is the cluster-total R of
    the grid that came out of the forward transform."""
    from oracle.oracle_cf import CfState
    j = synthetic_job()
    m = build_reflection_model(j, 32)
    st = CfState(m, model_initial_grid(m, 32, 7), 1.1, 0.0, 7)
    F0 = st.F.copy()
    R = st.cycle()
    rho = np.fft.ifftn(F0.reshape(32, 32, 32)).ravel().real
    assert abs(st.last_delta - 1.1 * rho.std()) <= 1e-12 * rho.std()
    flipped = np.where(rho < st.last_delta, -rho, rho)
    Ff = np.fft.fftn(flipped.reshape(32, 32, 32)).ravel()
    num = den = 0.0
    for c in range(m['n_clusters']):
        s, n = m['cluster_orbit_start'][c], m['cluster_n_orbits'][c]
        tot = 0.0
        for o in range(s, s + n):
            idx = m['orbit_idx'][m['orbit_start'][o]:m['orbit_start'][o] + m['orbit_count'][o]] & IDX_MASK
            tot += np.sum(np.abs(Ff[idx]) ** 2)
        num += abs(math.sqrt(tot) - math.sqrt(m['cluster_obs_i'][c]))
        den += math.sqrt(m['cluster_obs_i'][c])
    assert abs(R - num / den) <= 1e-12
    for o in range(m['n_orbits']):
        idx = m['orbit_idx'][m['orbit_start'][o]:m['orbit_start'][o] + m['orbit_count'][o]] & IDX_MASK
        a = np.abs(st.F[idx])
        assert np.max(a) - np.min(a) <= 1e-9 * max(1.0, np.max(a))
    assert np.all(st.F[m['orbit_idx'][m['n_members']:]] == 0) and st.F[0] == 0


def test_oracle_converges_on_the_synthetic_structure():
    """P1-style flipping (sym_lambda 0) on exact, unoverlapped intensities of
    the synthetic P2_1/c structure at 32^3 drops R from 0.66 to below 0.1 in
    150 cycles; the best grid is the one the best R was reached on."""
    from oracle.oracle_cf import CfState
    j = synthetic_job(overlap_tol=0.0)
    m = build_reflection_model(j, 32)
    st = CfState(m, model_initial_grid(m, 32, 543), 1.1, 0.0, 543)
    R = [st.cycle() for _ in range(150)]
    assert R[0] > 0.5 and min(R) < 0.1 and st.best_r == min(R)
