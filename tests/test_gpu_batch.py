"""Batched searches in one persistent launch against the same searches run
one launch each: the ladders are independent and every draw is keyed by
(search, replica, generation), so the results must be bit-identical."""
import numpy as np
import pytest

from powder6_b200.batch import WyckoffBatch, autotune, reset, run_batched, setup_searches
from powder6_b200.swarm_wyckoff import SW_DEFAULTS
from powder6_b200.workloads import batched_problems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def items():
    its = batched_problems(6, seed=3)
    for it in its:
        it.replicas = min(it.replicas, 256)
    return its


def states(setup):
    return [s.read_state() for s in setup.sessions]


def separate(items, gens):
    setup = setup_searches(items, gens, seed=5)
    reset(setup)
    for s in setup.sessions:
        s.run(0, gens, int(SW_DEFAULTS['swapEvery']), True)
        s.synchronize(120)
    out = states(setup)
    for s in setup.sessions:
        s.close()
    return out


@pytest.mark.parametrize('use_graph,order', [(False, 0), (True, 1)])
def test_batch_is_bit_identical_to_separate_launches(items, use_graph, order):
    gens = 120
    ref = separate(items, gens)
    setup = setup_searches(items, gens, seed=5)
    try:
        with WyckoffBatch(setup.sessions) as b:
            b.set_launch(0, order)
            for rep in range(2):                       # a second run (graph replay) from the same start
                reset(setup)
                b.run([0] * len(items), [gens] * len(items), int(SW_DEFAULTS['swapEvery']), True, use_graph)
                b.synchronize()
                got = states(setup)
                for (p0, b0, s0), (p1, b1, s1) in zip(ref, got):
                    assert np.array_equal(p0, p1) and np.array_equal(b0, b1)
                    assert s0.tobytes() == s1.tobytes()
            assert b.query()['launches'] == 2
    finally:
        for s in setup.sessions:
            s.close()


def test_autotune_and_run(items):
    r = run_batched(items, generations=100, seed=2, tune=True)
    t = r['tuning']
    assert 1 <= t['ctas_per_sm'] <= r['query']['max_ctas_per_sm'] and t['order'] in (0, 1)
    assert len(t['trials']) == 2 * r['query']['max_ctas_per_sm']
    assert r['ms'] > 0 and len(r['results']) == len(items)
    assert all(np.isfinite(x['best_cc']) and 0 <= x['best_cc'] <= 1 for x in r['results'])
