"""Particle budget over Wyckoff assignments: weighting by free parameters,
waves and successive halving (js/wyckoff_assign.js:1188-1278), restated on
the host, checked against hand-computed allocations."""
import math

import numpy as np

from powder6_b200.swarm_wyckoff import (allocate_waves, assignment_dims, assignments_per_wave, prune_assignments,
                                        weighted_assign)
from powder6_b200.workloads import wyckoff_problem

ALTERNATIVES = (
    (('Pb', '4c'), ('S', '4c'), ('O', '8d'), ('O', '8d')),
    (('Pb', '4a'), ('S', '4c'), ('O', '4c'), ('O', '4c'), ('O', '8d')),
    (('Pb', '4b'), ('S', '4c'), ('O', '4c'), ('O', '4c'), ('O', '8d')),
    (('Pb', '4c'), ('S', '4a'), ('O', '4c'), ('O', '4c'), ('O', '8d')),
    (('Pb', '4c'), ('S', '4b'), ('O', '8d'), ('O', '8d')),
)


def counts(a, ids):
    return [int(np.sum(a == i)) for i in ids]


def test_weighted_assign_floor_surplus_and_remainder():
    # floor 24 each, surplus 440 split 1 : 2 : 5 exactly
    a = weighted_assign([0, 1, 2], 512, 24, [1, 2, 5])
    assert counts(a, [0, 1, 2]) == [24 + 55, 24 + 110, 24 + 275]
    # contiguous blocks in the order of ids
    assert np.all(np.diff(a.astype(np.int64)) >= 0)
    # equal weights: 24 + 9 each, the one left over to the first of the (tied) largest
    assert counts(weighted_assign([0, 1, 2], 100, 24, None), [0, 1, 2]) == [34, 33, 33]
    # more assignments than the floor allows: the floor shrinks to n // len(ids)
    a = weighted_assign(list(range(10)), 100, 24, [1] * 10)
    assert counts(a, range(10)) == [10] * 10
    # ids out of order keep their order; weights are looked up by id (id 2 weighs 1, id 0 weighs 3)
    a = weighted_assign([2, 0], 60, 24, [3, 1, 1])
    assert list(a[:27]) == [2] * 27 and list(a[27:]) == [0] * 33


def test_prune_keeps_the_better_half_and_at_least_four():
    best = {0: 0.9, 1: 0.5, 2: 0.7, 3: 0.1, 4: 0.8, 5: 0.3, 6: 0.6}
    assert prune_assignments(list(range(7)), best) == [0, 4, 2, 6]          # ceil(7 / 2) = 4
    assert prune_assignments(list(range(5)), best) == [0, 4, 2, 1]          # max(4, 3)
    assert prune_assignments([3, 5, 1], best) == [1, 5, 3]                  # fewer than four: all, ranked
    ids = list(range(10))
    kept = prune_assignments(ids, {a: float(a) for a in ids if a != 9})
    assert kept == [8, 7, 6, 5, 4]                                          # no best: ranked last
    assert len(prune_assignments(ids, {}, 0.3, 2)) == math.ceil(10 * 0.3)


def test_waves_hold_room_to_weight():
    assert assignments_per_wave(512, 24, True) == 10
    assert assignments_per_wave(512, 24, False) == 21
    assert assignments_per_wave(16, 24, True) == 1
    waves = allocate_waves(range(21), 512, 24, [1] * 21)
    assert [len(w) for w in waves] == [10, 10, 1] and waves[2] == [20]


def test_assignment_dims_count_free_parameters():
    P = wyckoff_problem(seed=1, extra_assignments=ALTERNATIVES)
    # 4c has x, z free; 8d x, y, z; 4a and 4b none
    assert assignment_dims(P) == [11, 10, 9, 9, 9, 8]
