"""Wyckoff trial kernel on the GPU, through the C ABI, against the FP64 oracle.

Tolerances (stated per test): the fitness cc = 1 - wR2 and the per-reflection
mult |F|^2 are FP32 arithmetic on exactly reduced integer phases; the oracle
is FP64.  Orbit expansion and proposals on the Wyckoff subspace are integer
arithmetic and are compared bit for bit."""
import dataclasses
import math

import numpy as np
import pytest

from powder6_b200 import _lib
from powder6_b200.swarm_wyckoff import (STATE_DTYPE, WyckoffSession, build_ladders, initial_state, project_all,
                                        run_wyckoff_search, schedule)
from powder6_b200.workloads import mulberry32, wyckoff_problem

pytestmark = pytest.mark.gpu

TWO32 = 2.0 ** 32


def to_fixed(x):
    f = np.asarray(x, dtype=np.float64)
    f = f - np.floor(f)
    v = np.floor(f * TWO32 + 0.5)
    v[v >= TWO32] -= TWO32
    return v.astype(np.uint64).astype(np.uint32)


def trans_fixed(t):
    s = t * 24.0
    r = math.floor(s + 0.5)
    assert abs(s - r) < 1e-4
    n = int(r) % 24
    return (n * 2 ** 32 + 12) // 24


def random_positions(P, n, seed):
    rng = np.random.default_rng(seed)
    assign = np.zeros(n, dtype=np.uint32)
    pos = project_all(P, rng.random(n * P.max_sites * 3).astype(np.float32), assign)
    return to_fixed(pos.astype(np.float64)), assign


def oracle_cc_pen(O, P, X_sites, n_groups, pen_scale, n_rules=0, slots=64, geom_slots=1):
    """FP64 fitness and penalty of already-projected fixed-point site coordinates."""
    x = X_sites.astype(np.float64) / TWO32
    gp = P.tables.gen_pack[:P.n_tot]
    cc, sums = O.wy_fitness_projected(x, gp, P.sym_packed, P.refl.group_meta, n_groups, 4, P.refl.refl_pack,
                                      P.f_tab, P.n_elem, P.centro)
    geom = O.make_geom(P.orth, P.xform, P.min_image_shell, 1, P.pen_clash, P.pen_bond, P.pen_coord, P.pen_geom,
                       pen_scale)
    pen = O.wy_penalty(x, gp, P.sym_packed, P.n_elem, P.restraints.tables, P.restraints.r_min_off,
                       P.restraints.rule_off, P.restraints.n_rules, slots, geom_slots, geom)
    return cc, pen, sums


def icalc_fp64(P, X_sites):
    """mult |F|^2 per reflection, FP64, from fixed-point sites (the oracle's arithmetic)."""
    x = X_sites.astype(np.float64) / TWO32
    ms = P.max_sites
    gp = P.tables.gen_pack[:P.n_tot].astype(np.int64)
    site, op, ty, skip = gp & 0xFF, (gp >> 8) & 0xFFF, (gp >> 20) & 0xF, (gp >> 24) & 1
    sym = P.sym_packed.astype(np.float64).reshape(-1, 12)
    g = np.einsum('aij,aj->ai', sym[op, :9].reshape(-1, 3, 3), x.reshape(ms, 3)[site]) + sym[op, 9:]
    g = g[skip == 0]
    ty = ty[skip == 0]
    pk = P.refl.refl_pack[0::2].astype(np.int64)
    hkl = np.stack([(pk & 0x3FF) - 512, ((pk >> 10) & 0x3FF) - 512, ((pk >> 20) & 0x3FF) - 512], 1)
    q = hkl @ g.T
    f = P.f_tab.astype(np.float64).reshape(-1, P.n_elem)[:, ty]
    F = (f * np.exp(2j * np.pi * (q - np.floor(q)))).sum(1)
    return P.refl.refl_pack[1::2] * np.abs(F) ** 2


@pytest.fixture(scope='module')
def prob():
    return wyckoff_problem(seed=1)


def test_philox_device_known_answer():
    lib = _lib.load()
    for ctr, key, exp in [([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
                          ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
                           [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1])]:
        c = np.array(ctr, dtype=np.uint32)
        k = np.array(key, dtype=np.uint32)
        o = np.zeros(4, dtype=np.uint32)
        _lib.check(lib.p6_philox_device(_lib.ptr(c), _lib.ptr(k), _lib.ptr(o)))
        assert list(o) == exp


def test_orbit_expansion_bit_exact(prob, oracle):
    P = prob
    n = 64
    X, assign = random_positions(P, n, 3)
    with WyckoffSession(P, n) as s:
        s.write_positions_fixed(X)
        rint = np.array([o.r for o in P.group.ops], dtype=np.int32).reshape(-1)
        tf = np.array([[trans_fixed(float(v)) for v in P.sym_packed.reshape(-1, 12)[o, 9:]]
                       for o in range(len(P.group.ops))], dtype=np.uint64).astype(np.uint32).reshape(-1)
        for p in (0, 17, 63):
            got = s.debug_expand(p)
            sites = X[p * P.max_sites * 3:(p + 1) * P.max_sites * 3]
            want = oracle.expand_fixed(sites, P.tables.gen_pack[:P.n_tot], rint, tf)
            assert np.array_equal(got, want)


CHI2 = lambda sums: 1.0 - sums[2] ** 2 / (sums[0] * sums[1])   # grouped wR2^2 after the best scale


@pytest.mark.parametrize('cos_mode,cc_tol,ic_tol,chi2_tol', [(0, 2e-6, 2e-4, None), (1, 5e-7, 5e-6, None),
                                                              (2, 1e-7, 1e-5, 1e-6)])
def test_evaluation_parity(prob, oracle, cos_mode, cc_tol, ic_tol, chi2_tol):
    """cc within cc_tol (absolute, on a [0, 1] fitness), penalty within 1e-5
    relative, and mult |F|^2 within ic_tol relative to the largest reflection
    of each structure (FP32 sum of FP32 cosines for modes 0 and 1, the
    factored FP64 evaluation for mode 2, vs FP64).  For the factored mode the
    device's FP64 fitness sums give the chi^2-like 1 - cc^2 (wR2^2 after the
    best scale) of every replica, random and true structures alike, within
    chi2_tol relative of the FP64 oracle's."""
    P = prob
    n = 256
    X, assign = random_positions(P, n, 5 + cos_mode)
    # put the first particles on the true structure and close to it
    tx = to_fixed(P.true_coords)
    X[:P.max_sites * 3] = tx
    with WyckoffSession(P, n, cos_mode=cos_mode) as s:
        s.write_positions_fixed(X)
        s.set_trace(True)
        worst_cc = worst_ic = worst_pen = worst_chi = 0.0
        for nga, scale in ((P.refl.n_groups, 1.0), (max(8, P.refl.n_groups // 4), 2.5)):
            s.set_params(nga, scale)
            s.dispatch(None, mcmc=False)
            s.synchronize(60)
            _, _, st = s.read_state()
            ic = s.read_trace_ic()
            dsums = s.read_trace_sums()
            for p in range(n):
                sites = X[p * P.max_sites * 3:(p + 1) * P.max_sites * 3]
                cc, pen, sums = oracle_cc_pen(oracle, P, sites, nga, scale)
                worst_chi = max(worst_chi, abs(CHI2(dsums[p]) - CHI2(sums)) / CHI2(sums))
                worst_cc = max(worst_cc, abs(float(st['cc'][p]) - cc))
                worst_pen = max(worst_pen, abs(float(st['pen'][p]) * scale - pen) / max(1.0, pen))
                assert abs(float(st['fit'][p]) - (cc - pen)) < cc_tol + 1e-5 * max(1.0, pen)
                if nga == P.refl.n_groups and p < 32:
                    ref = icalc_fp64(P, sites)
                    worst_ic = max(worst_ic, float(np.max(np.abs(ic[p] - ref)) / ref.max()))
        print(f'cos_mode {cos_mode}: max |dcc| {worst_cc:.3e}, max rel |d mult F^2| {worst_ic:.3e}, '
              f'max rel dpen {worst_pen:.3e}, max rel d(1 - cc^2) {worst_chi:.3e}')
        assert worst_cc <= cc_tol
        if chi2_tol is not None:
            assert worst_chi <= chi2_tol
        assert worst_ic <= ic_tol
        assert worst_pen <= 1e-5
        assert float(st['cc'][0]) > 0.95


def _pair_cases():
    hexa = {'a': 5.0, 'b': 5.0, 'c': 14.0, 'alpha': 90.0, 'beta': 90.0, 'gamma': 120.0}
    mono = {'a': 9.0, 'b': 6.0, 'c': 8.0, 'alpha': 90.0, 'beta': 105.0, 'gamma': 90.0}
    return {
        # Pnma evaluated with the complex sums: the pairs' sines must cancel
        'pnma-complex': lambda: dataclasses.replace(wyckoff_problem(seed=1), centro=False),
        # R-3m (hexagonal axes): translations of 1/3 and 2/3 and rhombohedral centring
        'r-3m': lambda: wyckoff_problem(seed=3, group_number=166, cell=hexa, composition=(('Ti', 6), ('O', 18)),
                                        sites=(('Ti', '6c'), ('O', '18h')), dmin=1.3, true_min_contact=1.2,
                                        contact_attempts=200),
        # C2/c: C centring, a general and a special position
        'c2/c': lambda: wyckoff_problem(seed=3, group_number=15, cell=mono, composition=(('S', 8), ('O', 4)),
                                        sites=(('S', '8f'), ('O', '4e')), dmin=1.3, true_min_contact=1.2,
                                        contact_attempts=200),
    }


@pytest.mark.parametrize('case', ['pnma-complex', 'r-3m', 'c2/c'])
def test_inversion_pair_evaluation_parity(oracle, case):
    """Images related by the inversion centre are summed once with weight 2
    (sines cancelled); the fitness still matches the FP64 oracle's sum over
    every image: |dcc| <= 2e-6 and mult |F|^2 within 2e-4 of the largest
    reflection (SFU cosines), on centred cells, fractional translations of
    1/3 and the complex-sum path.  The clash penalty, summed from each
    site's representative with weight m_s / 2, matches the oracle's sum over
    all pairs within 1e-5 relative on random (clashing) structures."""
    P = _pair_cases()[case]()
    n = 128
    X, _ = random_positions(P, n, 21)
    with WyckoffSession(P, n, cos_mode=0) as s:
        s.write_positions_fixed(X)
        s.set_trace(True)
        s.set_params(P.refl.n_groups, 1.0)
        s.dispatch(None, mcmc=False)
        s.synchronize(60)
        _, _, st = s.read_state()
        ic = s.read_trace_ic()
    worst_cc = worst_ic = worst_pen = 0.0
    clashing = 0
    for p in range(n):
        sites = X[p * P.max_sites * 3:(p + 1) * P.max_sites * 3]
        cc, pen, _ = oracle_cc_pen(oracle, P, sites, P.refl.n_groups, 1.0)
        worst_cc = max(worst_cc, abs(float(st['cc'][p]) - cc))
        worst_pen = max(worst_pen, abs(float(st['pen'][p]) - pen) / max(1.0, pen))
        clashing += pen > 0
        if p < 32:
            ref = icalc_fp64(P, sites)
            worst_ic = max(worst_ic, float(np.max(np.abs(ic[p] - ref)) / ref.max()))
    print(f'{case}: max |dcc| {worst_cc:.3e}, max rel |d mult F^2| {worst_ic:.3e}, max rel dpen {worst_pen:.3e}, '
          f'{clashing}/{n} with clashes')
    assert worst_cc <= 2e-6
    assert worst_ic <= 2e-4
    assert worst_pen <= 1e-5
    assert clashing >= n // 16


def test_mcmc_step_parity_and_proposals(prob, oracle):
    """One generation with tracing: each proposal is re-scored by the oracle,
    the acceptance follows the kernel's own rule, unmoved sites are bit-identical,
    moved sites lie on their Wyckoff subspace, and the state update matches."""
    P = prob
    n = 512
    X, assign = random_positions(P, n, 9)
    rnd = mulberry32(4)
    temps = np.full(n, 0.01, dtype=np.float32)
    st0 = initial_state(n, temps, rnd)
    with WyckoffSession(P, n, run_key=77) as s:
        s.write_positions_fixed(X)
        s.set_params(P.refl.n_groups, 1.0)
        s.dispatch(None, mcmc=False)                       # measure the current state first
        s.synchronize(60)
        _, _, st = s.read_state()
        st['step_size'] = 0.05
        st['temp'] = temps
        st['seed'] = st0['seed']
        st['best_fit'] = -1e30
        cur_f = np.zeros(n * P.max_sites * 3, dtype=np.float32)
        # restore exact coordinates after sync_state (which takes float32) by rewriting fixed point
        s.sync_state(cur_f, st)
        s.write_positions_fixed(X)
        s.set_trace(True)
        s.set_params(P.refl.n_groups, 1.0)
        s.dispatch(None, mcmc=True)
        s.synchronize(60)
        props, rec = s.read_trace()
        after, best = s.read_positions_fixed()
        _, _, st1 = s.read_state()
    ms3 = P.max_sites * 3
    n_single = n_coll = 0
    worst = 0.0
    for p in range(n):
        x0 = X[p * ms3:(p + 1) * ms3].reshape(-1, 3)
        x1 = props[p * ms3:(p + 1) * ms3].reshape(-1, 3)
        moved = [i for i in range(P.max_sites) if not np.array_equal(x0[i], x1[i])]
        if len(moved) == 1:
            n_single += 1
        elif len(moved) > 1:
            n_coll += 1
        for i in range(P.max_sites):
            w = P.assignments[0].sites[i].w
            if w.triplet == 'x,1/4,z':
                assert x1[i][1] == 2 ** 30                   # y pinned exactly to 1/4
        cc, pen, _ = oracle_cc_pen(oracle, P, props[p * ms3:(p + 1) * ms3], P.refl.n_groups, 1.0)
        f_new, cc_g, pen_g, u, acc, f_old, temp, step_before = rec[p]
        worst = max(worst, abs(cc_g - cc))
        assert abs(pen_g - pen) <= 1e-5 * max(1.0, pen)
        prob_acc = math.exp(min(0.0, f_new - f_old) / max(temp, 1e-9))
        rule = f_new >= f_old or u < prob_acc
        if abs(u - prob_acc) > 1e-5:                          # float vs double exp at the boundary
            assert bool(acc) == rule
        state_x = after[p * ms3:(p + 1) * ms3]
        assert np.array_equal(state_x, props[p * ms3:(p + 1) * ms3] if acc else X[p * ms3:(p + 1) * ms3])
        want_step = step_before * (s.adapt['STEP_UP'] if acc else s.adapt['STEP_DOWN'])
        want_step = min(max(want_step, s.adapt['STEP_MIN']), s.adapt['STEP_MAX'])
        assert abs(float(st1['step_size'][p]) - want_step) < 1e-6 * want_step
        assert int(st1['accepted'][p]) == int(st['accepted'][p]) + int(acc)
    assert worst <= 2e-6
    # 3/4 single-site proposals, binomial tolerance
    frac = n_single / max(1, n_single + n_coll)
    assert 0.65 < frac < 0.85, frac


def test_fused_run_is_deterministic_and_exchanges(prob):
    P = prob
    n = 512
    results = []
    for _ in range(2):
        rnd = mulberry32(99)
        assign = np.zeros(n, dtype=np.uint32)
        with WyckoffSession(P, n, run_key=12345) as s:
            s.set_assign(assign)
            lad, temps = build_ladders(assign)
            s.set_ladders(lad, 8)
            g, pen = schedule(300, P.refl.n_groups)
            s.set_schedule(g, pen)
            pos = project_all(P, np.array([rnd() for _ in range(n * P.max_sites * 3)], dtype=np.float32), assign)
            st = initial_state(n, temps, rnd)
            s.sync_state(pos, st)
            s.run(0, 150, 10, True)
            s.run(150, 150, 10, bool(g[150] != g[149]))
            s.synchronize(120)
            cur, best = s.read_positions_fixed()
            _, _, st1 = s.read_state()
            results.append((cur.copy(), best.copy(), st1.copy()))
    (c0, b0, s0), (c1, b1, s1) = results
    assert np.array_equal(c0, c1) and np.array_equal(b0, b1)
    assert np.array_equal(s0.view(np.uint32), s1.view(np.uint32))
    assert np.all((s0['cc'] >= 0) & (s0['cc'] <= 1))
    assert np.all(s0['best_fit'] > -1e29)
    acc = s0['accepted'].sum() / (n * 300)
    assert 0.02 < acc < 0.9


def test_search_recovers_the_true_structure(prob):
    """wyckoff-search.js:82-84: the winner's GPU fitness agrees with the CPU
    re-score to 1e-3; and on this synthetic problem the search finds the truth."""
    P = prob
    res = run_wyckoff_search(P, num_particles=1024, generations=1500, restarts=1, seed=20261026, chunk=500)
    assert res.cpu_check['delta'] <= 1e-3
    assert res.best_cc >= 0.95, res.best_cc
    assert res.launches >= 3


def test_quench_only_improves_and_reports_time_to_target(prob):
    """quench (js/swarm_wyckoff.js:2013-2100): from a short search, the greedy
    quench at full resolution never loses the re-measured start, its winner
    re-scores on the CPU, and time_to_target is reported when reached."""
    P = prob
    short = run_wyckoff_search(P, num_particles=512, generations=300, seed=7, chunk=100, do_quench=False)
    res = run_wyckoff_search(P, num_particles=512, generations=300, seed=7, chunk=100, do_quench=True,
                             target_cc=short.best_cc - 0.05)
    q = res.quench
    assert q and q['ms'] > 0
    assert res.best_cc >= q['best_before'] - 2e-3       # the start is re-measured at full resolution
    assert res.cpu_check['delta'] <= 1e-3
    assert res.time_to_target is not None and res.time_to_target <= res.wall_s


def test_quench_accepts_improvements_only(prob):
    """In quench mode every accepted proposal raised the fitness, and the step
    widths stay where the search left them (no adaptation)."""
    from powder6_b200.swarm_wyckoff import build_ladders, initial_state, project_all, quench_schedule
    from powder6_b200.workloads import mulberry32
    P = prob
    n = 256
    rnd = mulberry32(5)
    with WyckoffSession(P, n) as s:
        assign = np.zeros(n, dtype=np.uint32)
        s.set_assign(assign)
        ladders, temps = build_ladders(assign)
        s.set_ladders(ladders, 8)
        pos = project_all(P, np.array([rnd() for _ in range(n * s.coords_per_particle)], dtype=np.float32), assign)
        st0 = initial_state(n, temps, rnd)
        s.sync_state(pos, st0)
        sd = quench_schedule()[:50]
        s.set_schedule(np.full(50, P.refl.n_groups, dtype=np.int32), np.full(50, 4.0, dtype=np.float32))
        s.set_quench(sd)
        s.set_trace(True)
        s.run(0, 50, 0, True)
        s.synchronize(60)
        _, rec = s.read_trace()
        _, _, st = s.read_state()
        s.set_quench(None)
    rec = rec.reshape(n, 8)
    acc = rec[:, 4] > 0.5
    assert np.all(rec[acc, 0] > rec[acc, 5])
    assert np.all(st['step_size'] == st0['step_size'])
    assert st['accepted'].sum() > 0


def test_restraint_rules_parity(oracle):
    """Counted shells, shapes and nearest-neighbour rules (the 64-slot variant)."""
    P = wyckoff_problem(seed=2, windows=[{'a': 'S', 'b': 'O', 'count': 4, 'dmin': 1.35, 'dmax': 1.65,
                                          'geometry': 'tetrahedron'},
                                         {'a': 'Pb', 'b': 'O', 'dmax': 3.2}])
    n = 128
    X, assign = random_positions(P, n, 21)
    with WyckoffSession(P, n) as s:
        s.write_positions_fixed(X)
        s.set_params(P.refl.n_groups, 1.7)
        s.dispatch(None, mcmc=False)
        s.synchronize(60)
        _, _, st = s.read_state()
    worst = 0.0
    for p in range(n):
        sites = X[p * P.max_sites * 3:(p + 1) * P.max_sites * 3]
        cc, pen, _ = oracle_cc_pen(oracle, P, sites, P.refl.n_groups, 1.7, P.restraints.n_rules, 64, 64)
        worst = max(worst, abs(float(st['pen'][p]) * 1.7 - pen) / max(1.0, pen))
    assert worst <= 2e-5, worst


def test_synchronize_deadline_and_recovery(prob):
    """A host wait that runs out returns TIMEOUT and leaves the session usable."""
    P = prob
    n = 4096
    with WyckoffSession(P, n) as s:
        assign = np.zeros(n, dtype=np.uint32)
        lad, temps = build_ladders(assign)
        s.set_ladders(lad, 8)
        g, pen = schedule(2000, P.refl.n_groups)
        s.set_schedule(g, pen)
        s.run(0, 2000, 10, True)
        with pytest.raises(_lib.P6Error) as e:
            s.synchronize(1e-6)
        assert e.value.status == 'TIMEOUT'
        s.synchronize(120)
        _, _, st = s.read_state()
        assert np.isfinite(st['fit']).all()


def test_argument_errors_are_reported():
    P = wyckoff_problem(seed=1)
    with pytest.raises(_lib.P6Error) as e:
        WyckoffSession(P, 0)
    assert e.value.status == 'INVALID_ARG'
    with WyckoffSession(P, 16) as s:
        with pytest.raises(_lib.P6Error) as e:
            s.set_assign(np.full(16, 3, dtype=np.uint32))
        assert e.value.status == 'INVALID_ARG'
        with pytest.raises(_lib.P6Error):
            s.run(0, 10, 10)                                  # no ladders yet


def _fused(P, n, gens, incremental, cos_mode=0):
    rnd = mulberry32(314)
    assign = np.zeros(n, dtype=np.uint32)
    with WyckoffSession(P, n, run_key=2718, cos_mode=cos_mode, incremental=incremental) as s:
        assert s.query()['incremental'] == bool(incremental)
        s.set_assign(assign)
        lad, temps = build_ladders(assign)
        s.set_ladders(lad, 8)
        g, pen = schedule(gens, P.refl.n_groups)
        s.set_schedule(g, pen)
        pos = project_all(P, np.array([rnd() for _ in range(n * P.max_sites * 3)], dtype=np.float32), assign)
        s.sync_state(pos, initial_state(n, temps, rnd))
        half = gens // 2
        s.run(0, half, 10, True)
        s.run(half, gens - half, 10, bool(g[half] != g[half - 1]))
        s.synchronize(120)
        cur, best = s.read_positions_fixed()
        _, _, st = s.read_state()
    return cur, best, st


@pytest.mark.parametrize('cos_mode', [0, 1])
def test_incremental_site_sums_are_bit_identical_to_full_evaluation(prob, cos_mode):
    """The cached per-site sums are re-summed in site order, so a search with
    them follows exactly the trajectory of full re-evaluation, through the
    resolution ramp and the ladder exchanges."""
    P = prob
    a = _fused(P, 512, 400, 1, cos_mode)
    b = _fused(P, 512, 400, 0, cos_mode)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.array_equal(a[2].view(np.uint32), b[2].view(np.uint32))


PBSO4_ALTERNATIVES = (
    (('Pb', '4c'), ('S', '4c'), ('O', '8d'), ('O', '8d')),
    (('Pb', '4a'), ('S', '4c'), ('O', '4c'), ('O', '4c'), ('O', '8d')),
    (('Pb', '4b'), ('S', '4c'), ('O', '4c'), ('O', '4c'), ('O', '8d')),
    (('Pb', '4c'), ('S', '4a'), ('O', '4c'), ('O', '4c'), ('O', '8d')),
    (('Pb', '4c'), ('S', '4b'), ('O', '8d'), ('O', '8d')),
)


def test_prune_keeps_the_better_half_and_finds_the_true_assignment():
    """Six assignments of PbSO4 in Pnma (the true one first), replicas shared
    by free-parameter count: at generation 0.45 G the better four stay, the
    other two's replicas move to them with fresh coordinates and ladders,
    the retired assignments keep the bests they had, and the true assignment
    wins, cross-checked on the CPU."""
    from powder6_b200.swarm_wyckoff import run_wyckoff_search
    P = wyckoff_problem(seed=1, extra_assignments=PBSO4_ALTERNATIVES)
    res = run_wyckoff_search(P, num_particles=4096, generations=4000, seed=5)
    assert res.assignments == list(range(6))
    assert len(res.kept) == 4 and 0 in res.kept
    assert set(res.per_assignment) == set(range(6))
    assert res.best_assignment == 0 and res.best_cc > 0.9, (res.best_assignment, res.best_cc, res.per_assignment)
    assert res.cpu_check['delta'] < 1e-5


def test_search_over_the_enumerated_assignments_finds_the_true_one():
    """Enumeration, then search: the twelve deduplicated PbSO4 assignments
    (tetrahedral S kept off the inversion centres) share 4096 replicas by
    free-parameter count, the prune keeps the better half, and the true
    assignment wins with cc > 0.9."""
    from powder6_b200.swarm_wyckoff import run_wyckoff_search
    from test_wyckoff_assign import enumerated_pbso4_alternatives
    alts, _ = enumerated_pbso4_alternatives()
    P = wyckoff_problem(seed=1, extra_assignments=alts)
    res = run_wyckoff_search(P, num_particles=4096, generations=4000, seed=5)
    assert res.assignments == list(range(12)) and 0 in res.kept
    assert res.best_assignment == 0 and res.best_cc > 0.9, (res.best_assignment, res.best_cc, res.per_assignment)


def test_waves_cover_every_assignment():
    """256 replicas hold five assignments per wave: two waves, every
    assignment searched, the best over both reported."""
    from powder6_b200.swarm_wyckoff import run_wyckoff_waves
    P = wyckoff_problem(seed=1, extra_assignments=PBSO4_ALTERNATIVES)
    res = run_wyckoff_waves(P, num_particles=256, generations=300, seed=9, do_quench=False)
    assert sorted(res.assignments) == list(range(6))
    assert set(res.per_assignment) == set(range(6))
    assert res.best_cc == max(res.per_assignment.values()) or res.best_pen > 0


# ---------------------------------------------------------------------------
# Polyhedron moves (swarm_reflection.wgsl:425-576) against an FP64 restatement
# ---------------------------------------------------------------------------
def _philox_stream(oracle, seed, run_key, g, p):
    """The lane-0 Philox stream of the polyhedron move: counter (g, p, 0x7000 + block, 6)."""
    import ctypes as C
    lib = oracle.load()
    blk = 0
    while True:
        ctr = np.array([g, p, 0x7000 + blk, 6], dtype=np.uint32)
        key = np.array([seed, run_key], dtype=np.uint32)
        out = np.zeros(4, dtype=np.uint32)
        lib.p6o_philox(ctr.ctypes.data_as(C.c_void_p), key.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p))
        for w in out:
            yield int(w)
        blk += 1


class _Stream:
    def __init__(self, gen):
        self.gen = gen

    def uniform(self):
        return np.float32((next(self.gen) >> 8) * (1.0 / 16777216.0))

    def gaussian(self):
        a, b = next(self.gen), next(self.gen)
        u_open = ((a >> 8) + 1) / 16777216.0
        return math.sqrt(-2.0 * math.log(u_open)) * math.cos(2 * math.pi * ((b >> 8) / 16777216.0))


_SHAPES = {1: [(1, 0, 0), (-1, 0, 0)],
           2: [(1, 0, 0), (-0.5, math.sqrt(3) / 2, 0), (-0.5, -math.sqrt(3) / 2, 0)],
           3: [tuple(v / math.sqrt(3) for v in t) for t in ((1, 1, 1), (1, -1, -1), (-1, 1, -1), (-1, -1, 1))],
           4: [(1, 0, 0), (0, 1, 0), (-1, 0, 0), (0, -1, 0)],
           5: [(1, 0, 0), (0, 1, 0), (-1, 0, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]}


def _frame(a, b):
    e1 = a / np.linalg.norm(a)
    pv = b - np.dot(b, e1) * e1
    if np.linalg.norm(pv) < 1e-4:
        h = np.array([0.0, 1.0, 0.0]) if abs(e1[0]) > 0.9 else np.array([1.0, 0.0, 0.0])
        pv = h - np.dot(h, e1) * e1
    e2 = pv / np.linalg.norm(pv)
    return np.stack([e1, e2, np.cross(e1, e2)], axis=1)       # columns


def _poly_restated(P, sites_fx, rng, sd):
    """polyPropose in FP64: returns ({site: new fraction (3,)}, kind); empty when no move applies."""
    T = P.tables
    ms, nT = T.max_sites, T.n_tot
    gp = [int(w) for w in T.gen_pack[:nT]]
    sym = P.sym_packed.astype(np.float64).reshape(-1, 12)
    tb = P.restraints.tables
    rules = [tb[P.restraints.rule_off + 7 * k:P.restraints.rule_off + 7 * k + 7] for k in range(P.restraints.n_rules)]
    n_counted, k = 0, 0
    for r, rb in enumerate(rules):
        if int(rb[5]) != 0:
            n_counted += 1
            if rng.uniform() < np.float32(1.0) / np.float32(n_counted):
                k = r
    if n_counted == 0:
        return {}, None
    rb = rules[k]
    ta, tbt, rmin, rmax, nn, geom = int(rb[0]), int(rb[1]), max(float(rb[2]), 0.0), float(rb[3]), min(int(rb[4]), 12), int(rb[6])
    n_c, sc, seen = 0, ms, set()
    for w in gp:
        s = w & 0xFF
        if s >= ms or ((w >> 20) & 0xF) != ta or s in seen:
            continue
        seen.add(s)
        n_c += 1
        if rng.uniform() < np.float32(1.0) / np.float32(n_c):
            sc = s
    if sc >= ms or nn == 0:
        return {}, None
    X = sites_fx.reshape(ms, 3).astype(np.int64)
    xf = np.asarray(P.xform, dtype=np.float64).reshape(3, 3).round().astype(np.int64)
    orth = np.asarray(P.orth, dtype=np.float64).reshape(3, 3)
    inv = np.asarray(P.inv_orth, dtype=np.float64).reshape(3, 3)
    cands = []
    for w in gp:
        s = w & 0xFF
        if s >= ms or s == sc or ((w >> 20) & 0xF) != tbt:
            continue
        o = (w >> 8) & 0xFFF
        R = sym[o, :9].round().astype(np.int64).reshape(3, 3)
        t = np.array([trans_fixed(float(v)) for v in sym[o, 9:]], dtype=np.int64)
        img = (R @ X[s] + t) % 2 ** 32
        d = (img - X[sc]) % 2 ** 32
        d = np.where(d >= 2 ** 31, d - 2 ** 32, d)
        q = (xf @ d) % 2 ** 32
        q = np.where(q >= 2 ** 31, q - 2 ** 32, q) / 2.0 ** 32
        dv = orth @ q
        dist = float(np.linalg.norm(dv))
        if dist < 1e-4:
            continue
        cands.append((dist, len(cands), dv, s, o))
    cands.sort(key=lambda c: (c[0], c[1]))            # stable: the first found wins a tie
    shell = cands[:nn]
    if not shell:
        return {}, None
    kind = rng.uniform()
    shift = np.zeros(3)
    lv = [c[2] for c in shell]
    ld = [c[0] for c in shell]
    nv = [v.copy() for v in lv]
    if kind < np.float32(0.3333333):
        shift = np.array([rng.gaussian(), rng.gaussian(), rng.gaussian()]) * sd
    elif kind < np.float32(0.6666667):
        ax = np.array([rng.gaussian(), rng.gaussian(), rng.gaussian()])
        ax = ax / np.linalg.norm(ax) if np.linalg.norm(ax) >= 1e-6 else np.array([0.0, 0.0, 1.0])
        ang = rng.gaussian() * min(max(sd * 20.0, 0.05), 0.8)
        c, sn = math.cos(ang), math.sin(ang)
        nv = [v * c + np.cross(ax, v) * sn + ax * np.dot(ax, v) * (1 - c) for v in lv]
    else:
        mean = sum(ld) / len(ld) * (1 + 0.03 * rng.gaussian())
        dT = min(max(mean, max(rmin, 0.3)), rmax if rmax < 1e6 else mean)
        shape = [np.array(v) for v in _SHAPES.get(geom, [])]
        if len(shape) >= 2 and len(shell) >= 2:
            u0 = lv[0] / ld[0]
            c_ideal = float(np.dot(shape[0], shape[1]))
            errs = [abs(float(np.dot(u0, lv[m] / ld[m])) - c_ideal) for m in range(1, len(shell))]
            j1 = 1 + int(np.argmin(errs))
            Fa, Fi = _frame(u0, lv[j1]), _frame(shape[0], shape[1])
            used = {0, 1}
            for m in range(len(shell)):
                if m == 0:
                    vk = 0
                elif m == j1:
                    vk = 1
                else:
                    best, vk = -2.0, len(shape)
                    for qv in range(2, len(shape)):
                        if qv in used:
                            continue
                        dd = float(np.dot(Fa @ (Fi.T @ shape[qv]), lv[m] / ld[m]))
                        if dd > best:
                            best, vk = dd, qv
                    if vk < len(shape):
                        used.add(vk)
                nv[m] = (Fa @ (Fi.T @ shape[vk])) * dT if vk < len(shape) else lv[m] / ld[m] * dT
        else:
            nv = [v / d * dT for v, d in zip(lv, ld)]
    cf = X[sc] / 2.0 ** 32
    out = {}
    if kind < np.float32(0.3333333):
        out[sc] = cf + shift
    for (dist, _, _, s, o), v in zip(shell, nv):
        if s in out:
            continue
        dest = cf + inv @ v + shift
        R = sym[o, :9].reshape(3, 3)
        t = np.array([trans_fixed(float(x)) for x in sym[o, 9:]], dtype=np.float64) / 2.0 ** 32
        out[s] = np.linalg.solve(R, dest - t)
    label = 'translate' if kind < np.float32(0.3333333) else 'rotate' if kind < np.float32(0.6666667) else 'snap'
    return out, label


def test_polyhedron_moves_match_the_restatement(oracle):
    """polyProb = 1 on a P2_1/c problem (S and four O on general positions, a
    counted S-O rule with a tetrahedron): every replica's proposal, as traced,
    equals the FP64 restatement of the move with the same random stream --
    the moved sites within 2e-5 (fractional, mod 1), the others bit for bit --
    and all three kinds of move occur."""
    cell = {'a': 7.2, 'b': 8.9, 'c': 10.4, 'alpha': 90.0, 'beta': 103.0, 'gamma': 90.0}
    P = wyckoff_problem(seed=4, group_number=14, cell=cell, composition=(('S', 4), ('O', 16)),
                        sites=(('S', '4e'), ('O', '4e'), ('O', '4e'), ('O', '4e'), ('O', '4e')), dmin=1.4,
                        windows=[{'a': 'S', 'b': 'O', 'count': 4, 'dmin': 1.35, 'dmax': 1.65,
                                  'geometry': 'tetrahedron'}], true_min_contact=1.2, contact_attempts=200)
    n, run_key = 192, 4242
    X, _ = random_positions(P, n, 77)
    rnd = mulberry32(5)
    st0 = initial_state(n, np.full(n, 0.01, dtype=np.float32), rnd)
    ms3 = P.max_sites * 3
    with WyckoffSession(P, n, run_key=run_key, settings={'polyProb': 1.0}) as s:
        s.sync_state(np.zeros(n * ms3, dtype=np.float32), st0)
        s.write_positions_fixed(X)
        s.set_trace(True)
        s.set_params(P.refl.n_groups, 1.0)
        s.dispatch(None, mcmc=True)
        s.synchronize(60)
        props, rec = s.read_trace()
    kinds = set()
    worst = 0.0
    for p in range(n):
        x0 = X[p * ms3:(p + 1) * ms3]
        got = props[p * ms3:(p + 1) * ms3].reshape(-1, 3)
        gen = _philox_stream(oracle, int(st0['seed'][p]), run_key, 0, p)
        rng = _Stream(gen)
        assert rng.uniform() < 1.0
        sd = float(st0['step_size'][p])
        want, kind = _poly_restated(P, x0, rng, sd)
        assert want, p                                    # a counted rule and partners always exist here
        for si in range(P.max_sites):
            if si in want:
                d = got[si] / 2.0 ** 32 - want[si]
                d -= np.round(d)
                worst = max(worst, float(np.max(np.abs(d))))
            else:
                assert np.array_equal(got[si], x0.reshape(-1, 3)[si]), (p, si)
        kinds.add(kind)
    print(f'polyhedron moves: worst fractional difference {worst:.2e}, kinds {sorted(kinds)}')
    assert worst < 2e-5
    assert kinds == {'translate', 'rotate', 'snap'}


PBSO4_MANY = PBSO4_ALTERNATIVES + (
    (('Pb', '4c'), ('S', '4c'), ('O', '4c'), ('O', '4c'), ('O', '4c'), ('O', '4c')),
    (('Pb', '4a'), ('S', '4b'), ('O', '8d'), ('O', '8d')),
    (('Pb', '4b'), ('S', '4a'), ('O', '8d'), ('O', '8d')),
    (('Pb', '4c'), ('S', '4c'), ('O', '4a'), ('O', '4c'), ('O', '8d')),
    (('Pb', '4c'), ('S', '4c'), ('O', '4b'), ('O', '4c'), ('O', '8d')),
    (('Pb', '4a'), ('S', '4c'), ('O', '8d'), ('O', '8d')),
)


def test_screening_stage_keeps_the_best_two_waves():
    """Twelve assignments, 256 replicas (five per wave): three waves exceed the
    two full-search waves, so every assignment is screened for a tenth of the
    generations, re-scored at full resolution, and only the best ten (two
    waves) are searched in full, in the order of their scores; the true
    assignment is among them and wins."""
    from powder6_b200.swarm_wyckoff import run_wyckoff_waves
    P = wyckoff_problem(seed=1, extra_assignments=PBSO4_MANY)
    res = run_wyckoff_waves(P, num_particles=256, generations=2000, seed=3)
    assert set(res.screened) == set(range(12))
    order = sorted(res.screened, key=lambda A: -res.screened[A])
    assert res.assignments == order[:10]
    assert 0 in res.assignments
    assert res.best_assignment == 0, (res.best_assignment, res.per_assignment)


def test_tables_too_large_to_stage_are_read_from_global_memory(oracle):
    """6432 reflections in 632 groups: the staged tables and eight replica
    slices exceed a CTA's shared memory, so the tables are read from global
    memory; the fitness and penalty match the oracle as on the staged path
    (cc within 2e-6, penalty within 1e-5), and a short fused search runs."""
    cell = {'a': 16.96, 'b': 10.80, 'c': 13.92, 'alpha': 90.0, 'beta': 90.0, 'gamma': 90.0}
    P = wyckoff_problem(seed=1, cell=cell, dmin=0.6, true_min_contact=1.2, contact_attempts=200)
    assert P.refl.n_refl > 6000
    n = 64
    X, _ = random_positions(P, n, 31)
    X[:P.max_sites * 3] = to_fixed(P.true_coords)
    with WyckoffSession(P, n) as s:
        q = s.query()
        assert q['smem_bytes'] < P.refl.n_refl * 4 * 8 + 8 * 1024 * 8   # slices only, no staged tables
        s.write_positions_fixed(X)
        s.set_params(P.refl.n_groups, 1.0)
        s.dispatch(None, mcmc=False)
        s.synchronize(60)
        _, _, st = s.read_state()
        worst_cc = worst_pen = 0.0
        for p in range(n):
            sites = X[p * P.max_sites * 3:(p + 1) * P.max_sites * 3]
            cc, pen, _ = oracle_cc_pen(oracle, P, sites, P.refl.n_groups, 1.0)
            worst_cc = max(worst_cc, abs(float(st['cc'][p]) - cc))
            worst_pen = max(worst_pen, abs(float(st['pen'][p]) - pen) / max(1.0, pen))
        assert worst_cc <= 2e-6 and worst_pen <= 1e-5, (worst_cc, worst_pen)
        assert float(st['cc'][0]) > 0.9
    res = run_wyckoff_search(P, num_particles=256, generations=100, seed=2, do_quench=False)
    assert np.isfinite(res.best_cc) and res.cpu_check['delta'] < 1e-5


def test_ladders_on_two_cta_clusters_are_bit_identical(prob):
    """The fused search with each ladder of 8 on a cluster of two 4-warp CTAs
    (exchange energies in rank 0's shared memory, cross-CTA swaps through
    distributed shared memory) gives the same coordinates, bests and states,
    bit for bit, as the one-CTA ladder, with exchanges taking place."""
    P = prob
    n, G = 1024, 300
    outs = []
    for split in (1, 2):
        with WyckoffSession(P, n, run_key=91) as s:
            s.set_ladder_split(split)
            assign = np.zeros(n, dtype=np.uint32)
            s.set_assign(assign)
            ladders, temps = build_ladders(assign)
            s.set_ladders(ladders, 8)
            groups, pen = schedule(G, P.refl.n_groups)
            s.set_schedule(groups, pen)
            rnd = mulberry32(17)
            pos = project_all(P, np.array([rnd() for _ in range(n * s.coords_per_particle)], dtype=np.float32), assign)
            s.sync_state(pos, initial_state(n, temps, rnd))
            s.run(0, G, 10, True)
            s.synchronize(120)
            cur, best = s.read_positions_fixed()
            _, _, st = s.read_state()
            outs.append((cur, best, st.tobytes()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    assert outs[0][2] == outs[1][2]
    st = np.frombuffer(outs[1][2], dtype=STATE_DTYPE)
    assert np.max(st['best_cc']) > 0.5


def test_coordinate_refinement_matches_the_restatement(oracle):
    """Three perturbed PbSO4 structures refined together on the device (FP64
    intensities, analytic constrained Jacobian, normal equations; damping on
    the host) reach the FP64 restatement's coordinates within 1e-9 and its wR
    within 1e-10 relative, with the same convergence and accepted steps."""
    from powder6_b200.swarm_wyckoff import refine_coordinates
    P = wyckoff_problem(seed=1)
    x_true = P.true_coords.copy()
    starts = [x_true + np.random.default_rng(s).uniform(-0.003, 0.003, x_true.shape) for s in (3, 4, 5)]
    with WyckoffSession(P, 64) as s:
        out = refine_coordinates(s, np.stack(starts), [0, 0, 0])
    for i, x0 in enumerate(starts):
        xr, r0, r1, chi, steps, conv = oracle.wy_refine(P, 0, x0)
        d = out['coords'][i] - xr
        d -= np.round(d)
        print(f'structure {i}: max |dx| {float(np.max(np.abs(d))):.2e}, r {out["r"][i]:.10f} vs {r1:.10f}, '
              f'steps {out["iterations"][i]} vs {steps}')
        assert np.max(np.abs(d)) < 1e-9, (i, float(np.max(np.abs(d))))
        assert abs(out['r_start'][i] - r0) <= 1e-10 * r0
        assert abs(out['r'][i] - r1) <= 1e-10 * r1, (out['r'][i], r1)
        assert int(out['iterations'][i]) == steps and bool(out['converged'][i]) == conv
        assert out['r'][i] < 0.02


def test_search_then_refinement(prob):
    """A short search followed by the least-squares refinement of its best
    structure: the refined wR(F^2) is at most the search's and reaches the
    true structure's."""
    from powder6_b200.swarm_wyckoff import run_wyckoff_search
    res = run_wyckoff_search(prob, num_particles=2048, generations=2000, seed=21, refine=True)
    ref = res.refined[0]
    assert ref['converged'] and ref['r'] <= ref['r_start'] + 1e-12
    assert ref['r'] < 0.02


def test_worker_job_runs_on_the_device():
    """A 'wyckoff-search' job message through the worker protocol to the
    device search and back: the enumerated PbSO4 assignments are searched,
    the progress stream carries the best so far, the winner is re-scored on
    the CPU and refined, and the final message is wy-structure."""
    from powder6_b200.workloads import wyckoff_job
    from powder6_b200.wyckoff_worker import WyckoffWorker
    P = wyckoff_problem(seed=1)
    out = []
    w = WyckoffWorker(out.append, threaded=False)
    w.on_message(wyckoff_job(P, swarmParticles=4096, swarmIterations=4000, seed=5))
    kinds = [m['type'] for m in out]
    assert kinds[0] == 'wy-start' and kinds[-1] == 'wy-structure', [m.get('message') for m in out]
    prog = [m for m in out if m['type'] == 'wy-progress']
    assert len(prog) >= 10 and all(m['bestSites'] for m in prog)
    assert prog[-1]['generation'] == 4000 and prog[-1]['fraction'] == pytest.approx(1.0)
    res = out[-1]['results']
    sol = res['wyckoffResult']
    assert sol['cpuCheck']['delta'] < 1e-5
    assert res['refinement']['R'] <= res['refinement']['RStart'] + 1e-12
    assert sum(s['multiplicity'] for s in res['sites']) == 24
    print('worker found', sol['assignment'], 'cc', sol['searchCC'], 'R', res['refinement'])
