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
