"""The rigid-fragment search on the device (config 5 in direct space): the
device's parameter -> coordinate map against the oracle's FP64 restatement,
every state the search leaves is the fragment at its parameters (bonds and
angles intact), and a search from random placements finds the structure."""
import numpy as np
import pytest

from oracle import oracle as O
from powder6_b200.crystal import orth_matrix
from powder6_b200.fragment import (device_coords, fragment_problem, random_params, read_fragment_state,
                                   run_fragment_search, set_fragment)
from powder6_b200.swarm_wyckoff import WyckoffSession

pytestmark = pytest.mark.gpu
TWO32 = 2.0 ** 32


@pytest.fixture(scope='module')
def config5():
    return fragment_problem(seed=1)


def _frac_err(a, b):
    d = a - b
    d -= np.round(d)
    return np.abs(d)


def test_device_map_matches_the_oracle(config5):
    P, frag, truth = config5
    prm = random_params(np.random.default_rng(7), 64, len(frag.torsions))
    prm[0] = truth
    with WyckoffSession(P, 64) as s:
        set_fragment(s, frag)
        got = device_coords(s, frag, prm).astype(np.float64) / TWO32
    worst = 0.0
    for p, g in zip(prm, got):
        want = O.fragment_coords_fp64(frag.ref, [t[0] for t in frag.torsions], [t[1] for t in frag.torsions],
                                      frag.moving, frag.to_frac, p.astype(np.float32).astype(np.float64))
        worst = max(worst, float(np.max(_frac_err(g, want))))
    print(f'fragment map: max |frac error| {worst:.2e}')
    assert worst < 2e-6        # FP32 arithmetic on coordinates of up to ~8 A: about 1e-5 A


def test_search_keeps_the_fragment_and_refines_from_near_the_truth(config5):
    """4096 replicas start at the true placement perturbed (translation 0.02,
    orientation and torsions about 0.2 rad), where the full-resolution cc is
    near 0; 2000 generations at full resolution bring the best back above
    0.9.  Every replica's coordinates are the device map of its parameters
    and the winner's bond lengths hold."""
    P, frag, truth = config5
    orth = orth_matrix(P.cell).astype(np.float64).reshape(3, 3)
    n = 4096
    rng = np.random.default_rng(5)
    start = np.tile(truth, (n, 1))
    start[:, :3] += rng.normal(size=(n, 3)) * 0.02
    start[:, 7:13] += rng.normal(size=(n, 6)) * 0.2
    q = start[:, 3:7] + rng.normal(size=(n, 4)) * 0.06
    start[:, 3:7] = q / np.linalg.norm(q, axis=1, keepdims=True)
    with WyckoffSession(P, n, run_key=3) as s:
        res = run_fragment_search(P, frag, n, 2000, seed=3, chunk=500, session=s, do_quench=True, start=start,
                                  full_resolution=True)
        cur_fx, _ = s.read_positions_fixed()
        cur_prm, _ = read_fragment_state(s)
        cpp = s.coords_per_particle
        idx = np.arange(0, n, 97)
        mapped = device_coords(s, frag, cur_prm[idx]).reshape(len(idx), -1)
        assert np.array_equal(mapped, cur_fx.reshape(n, cpp)[idx, :frag.n_atoms * 3])
    f = res.best_coords[:frag.n_atoms * 3].reshape(-1, 3).astype(np.float64)
    for u, v in frag.bonds:
        e = f[u] - f[v]
        e -= np.round(e)
        assert abs(np.linalg.norm(orth @ e) - np.linalg.norm(frag.ref[u] - frag.ref[v])) < 1e-3
    print(f'fragment refinement from near the truth: best cc {res.best_cc:.4f}, {res.kernel_ms:.0f} ms on the device')
    assert res.best_cc > 0.9


def test_fragment_search_scored_on_the_pattern(config5):
    # the fragment's fitness as the pattern's chi^2 in Gram form: every replica's
    # 1 - Rwp after a short search equals the oracle's (FP64 intensities of the
    # device's coordinates, FP64 fitted-scale chi^2 over the dense pattern)
    from powder6_b200.profile_search import pattern_gram, profile_problem, set_session_pattern
    P, frag, _ = config5
    pp = profile_problem(P, seed=1)           # the dense pattern on the grid pattern_gram uses
    with WyckoffSession(P, 64, run_key=4) as s:
        set_session_pattern(s, pattern_gram(P, seed=1))
        run_fragment_search(P, frag, 64, 30, seed=4, chunk=30, session=s, do_quench=False, full_resolution=True)
        _, _, st = s.read_state()
        cur, _ = s.read_positions_fixed()
    cpp = P.tables.max_sites * 3
    x = cur.astype(np.float64).reshape(-1, cpp) / TWO32
    I = np.array([O.wy_reflection_intensities(P, 0, xi) for xi in x])
    chi, _, syy = O.profile_fitted_chi2(I, pp.profile_t, pp.yobs, pp.w)
    r = np.sqrt(chi / syy)
    err = np.abs((1.0 - st['cc'].astype(np.float64)) - r)
    print(f'fragment, Gram form: max |Rwp - Rwp64| {err.max():.2e} (Rwp {r.min():.3f}..{r.max():.3f})')
    assert np.all(err <= 1e-5 * r + 2e-7)


def test_fragment_parameters_follow_the_contraction_search(config5):
    # the fragment searched with the pattern's chi^2 from the split-BF16 contraction
    # (deferred acceptance): after accepted moves, bests and ladder exchanges every
    # replica's current and best coordinates are the device map of its current and
    # best parameters, bit for bit
    from powder6_b200._lib import check
    from powder6_b200.contraction import SPLIT3_BF16, ContractionSession
    from powder6_b200.profile_search import _ContractionInput, profile_problem
    from powder6_b200.swarm_wyckoff import SW_DEFAULTS, build_ladders, initial_state, schedule
    from powder6_b200.workloads import mulberry32
    from powder6_b200.fragment import fragment_coords
    P, frag, _ = config5
    pp = profile_problem(P, seed=1)
    n = 256
    with WyckoffSession(P, n, run_key=6) as s, ContractionSession(_ContractionInput(pp), max_replicas=n) as ct:
        ct.set_fitted(True)
        set_fragment(s, frag)
        cpp = s.coords_per_particle
        assign = np.zeros(n, dtype=np.uint32)
        s.set_assign(assign)
        ladders, temps = build_ladders(assign, 8, SW_DEFAULTS['tempCold'], SW_DEFAULTS['tempHot'])
        s.set_ladders(ladders, 8)
        groups, pen = schedule(60, P.refl.n_groups)
        groups[:] = P.refl.n_groups
        s.set_schedule(groups, pen)
        prm = random_params(np.random.default_rng(6), n, len(frag.torsions))
        pos = np.zeros((n, cpp), dtype=np.float32)
        for i in range(n):
            pos[i, :frag.n_atoms * 3] = fragment_coords(frag, prm[i]).reshape(-1)
        s.sync_state(pos.reshape(-1), initial_state(n, temps, mulberry32(6)))
        from powder6_b200.fragment import write_fragment_state
        write_fragment_state(s, prm)
        check(s.lib.p6_wy_profile_run(s.h, ct.h, SPLIT3_BF16, 0, 0, 10, 1, 0))
        check(s.lib.p6_wy_profile_run(s.h, ct.h, SPLIT3_BF16, 0, 60, 10, 0, 0))
        s.synchronize(120)
        cur_fx, best_fx = s.read_positions_fixed()
        cur_prm, best_prm = read_fragment_state(s)
        _, _, st = s.read_state()
        assert st['accepted'].sum() > 0
        assert np.any(np.abs(cur_prm - prm.astype(np.float32)) > 0)
        for fx, pr in ((cur_fx, cur_prm), (best_fx, best_prm)):
            mapped = device_coords(s, frag, pr).reshape(n, -1)
            assert np.array_equal(mapped, fx.reshape(n, cpp)[:, :frag.n_atoms * 3])
