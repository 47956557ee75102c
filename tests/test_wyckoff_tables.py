"""Assignment, restraint and schedule tables (js/wyckoff_assign.js:756-1187,
js/swarm_wyckoff.js:201-216, 934-938, 1784-1808)."""
import math

import numpy as np
import pytest

from powder6_b200.swarm_wyckoff import adaptation, build_ladders, project_all, schedule
from powder6_b200.symmetry import space_group
from powder6_b200.wyckoff_tables import (Assignment, Site, build_assignment_tables, build_restraint_tables,
                                         make_assignment, pack_sym_ops, project_sites)

CENTRED = {
    12: [[('A', '8j'), ('B', '8j')], [('A', '4i'), ('A', '4i'), ('B', '4g'), ('B', '4h')]],
    166: [[('A', '18h'), ('B', '18g')], [('A', '9e'), ('A', '9d'), ('B', '18f')]],
    225: [[('A', '32f'), ('B', '32f')], [('A', '8c'), ('A', '24d'), ('B', '24e'), ('B', '8c')],
          [('A', '4a'), ('A', '4b'), ('A', '24e'), ('B', '32f')]],
}


@pytest.mark.parametrize('number', sorted(CENTRED))
def test_centring_skip_gives_full_intensity(number):
    """regressions.test.cjs:1618-1645: one image per centring class gives
    |F_full|^2 = n_C^2 |F_skip|^2 for reflections the centring allows."""
    g = space_group(number)
    count = {12: 8, 166: 18, 225: 32}[number]
    demand = [{'element': 'A', 'count': count, 'z': 20}, {'element': 'B', 'count': count, 'z': 8}]
    lists = [make_assignment(g, demand, a) for a in CENTRED[number]]
    T = build_assignment_tables(lists, g, demand)
    nC = len(T.centring) + 1
    assert nC > 1
    for ai, A in enumerate(lists):
        skip = T.gen_skip[ai * T.n_tot:(ai + 1) * T.n_tot]
        assert int((skip == 0).sum()) == T.n_tot // nC
        pos = [s.w.project(0.11 + 0.07 * si, 0.23 + 0.05 * si, 0.37 + 0.03 * si) for si, s in enumerate(A.sites)]
        for h in ([1, 1, 1], [2, 0, 0], [2, 2, 0], [3, 1, 1], [1, 0, 1], [0, 0, 3], [1, 1, 0], [4, 2, 0]):
            if not all(abs(sum(h[i] * c[i] for i in range(3)) - round(sum(h[i] * c[i] for i in range(3)))) < 1e-6
                       for c in T.centring):
                continue
            fr = fi = gr = gi = 0.0
            for gidx in range(T.n_tot):
                o = g.ops[T.gen_op[ai * T.n_tot + gidx]]
                p = pos[T.gen_site[ai * T.n_tot + gidx]]
                f = 8 if T.gen_type[ai * T.n_tot + gidx] else 20
                q = [sum(o.r[3 * i + k] * p[k] for k in range(3)) + o.t_frac[i] for i in range(3)]
                ph = 2 * math.pi * sum(h[i] * q[i] for i in range(3))
                fr += f * math.cos(ph)
                fi += f * math.sin(ph)
                if not skip[gidx]:
                    gr += f * math.cos(ph)
                    gi += f * math.sin(ph)
            full = fr * fr + fi * fi
            assert abs(full - nC * nC * (gr * gr + gi * gi)) < 1e-9 * max(1, full), (number, h)
    assert (int(T.gen_pack[0]) >> 24) & 1 == int(T.gen_skip[0])


def test_gen_pack_layout_and_projectors():
    g = space_group(62)
    demand = [{'element': 'Pb', 'count': 4, 'z': 82}, {'element': 'S', 'count': 4, 'z': 16},
              {'element': 'O', 'count': 16, 'z': 8}]
    A = make_assignment(g, demand, [('Pb', '4c'), ('S', '4c'), ('O', '4c'), ('O', '4c'), ('O', '8d')])
    B = make_assignment(g, demand, [('Pb', '4c'), ('S', '4c'), ('O', '8d'), ('O', '8d')])
    T = build_assignment_tables([A, B], g, demand)
    assert T.n_tot == 24 and T.max_sites == 5 and list(T.site_count) == [5, 4]
    gp = T.gen_pack[:24]
    assert [int(v) & 0xFF for v in gp] == [0] * 4 + [1] * 4 + [2] * 4 + [3] * 4 + [4] * 8
    assert [(int(v) >> 20) & 0xF for v in gp] == [0] * 4 + [1] * 4 + [2] * 16
    # 4c projector: (x, 1/4, z); unused site slot of B projects to zero
    b = (0 * 5 + 0) * 12
    assert list(T.site_proj[b:b + 12]) == [1, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0.25, 0]
    assert not np.any(T.site_proj[(1 * 5 + 4) * 12:(1 * 5 + 5) * 12])
    pos = np.random.default_rng(0).random(2 * 15).astype(np.float32)
    ref = pos.copy()
    project_sites(ref, 1, 1, T)
    got = project_all(type('P', (), {'tables': T})(), pos.copy(), np.array([0, 1]))
    assert np.allclose(got[15:], ref[15:], atol=1e-7)
    assert ref[15 + 4 * 3] == 0 and abs(ref[15 + 1] - 0.25) < 1e-7
    sym = pack_sym_ops(g.ops)
    assert sym.shape == (8 * 12,) and list(sym[:12]) == [1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0]


def test_capacity_checks():
    g = space_group(1)
    demand = [{'element': 'E%d' % i, 'count': 1, 'z': 6} for i in range(9)]
    A = make_assignment(g, demand, [('E%d' % i, '1a') for i in range(9)])
    with pytest.raises(ValueError, match='elements'):
        build_assignment_tables([A], g, demand)
    demand = [{'element': 'C', 'count': 33, 'z': 6}]
    A = make_assignment(g, demand, [('C', '1a')] * 33)
    with pytest.raises(ValueError, match='32'):
        build_assignment_tables([A], g, demand)


def test_restraint_tables_layout_and_rules():
    demand = [{'element': 'Pb', 'count': 4, 'z': 82}, {'element': 'S', 'count': 4, 'z': 16},
              {'element': 'O', 'count': 16, 'z': 8}]
    R = build_restraint_tables(demand, [{'a': 'S', 'b': 'O', 'count': 4, 'dmin': 1.35, 'dmax': 1.65,
                                         'geometry': 'tetrahedron'},
                                        {'a': 'Pb', 'b': 'O', 'dmax': 3.0}], min_contact=1.1)
    assert R.n_elem == 3 and R.r_min_off == 3 and R.rule_off == 12
    rmin = R.tables[3:12].reshape(3, 3)
    assert np.isclose(rmin[1, 2], 1.35) and np.isclose(rmin[2, 1], 1.35) and np.isclose(rmin[0, 0], 1.1)
    # counted rule (exact, tetrahedral) + the bare upper bound emitted both ways
    assert R.n_rules == 3 and R.slots_needed == 4 and R.geometry
    assert list(R.tables[12:19]) == pytest.approx([1, 2, 1.35, 1.65, 4, 1, 3])
    assert list(R.tables[19:26]) == pytest.approx([0, 2, 0, 3.0, 0, 0, 0])
    assert list(R.tables[26:33]) == pytest.approx([2, 0, 0, 3.0, 0, 0, 0])
    assert R.max_distance == pytest.approx(3.0)
    with pytest.raises(ValueError, match='tetrahedral|tetrahedron'):
        build_restraint_tables(demand, [{'a': 'S', 'b': 'O', 'count': 3, 'dmax': 1.6, 'geometry': 'tetrahedron'}])
    R0 = build_restraint_tables(demand, [])
    assert R0.n_rules == 0 and np.all(R0.tables[3:12] == 1.0)     # default contact floor 1.0 A
    assert np.all(build_restraint_tables(demand, [], min_contact=0).tables[3:12] == 0)


def test_adaptation_factors_and_validation():
    """wyckoff-adaptation.test.cjs:11-24: Robbins-Monro factors, bounds, and refusal."""
    s = {'stepMin': .001, 'stepMax': .25, 'stepInit': .04, 'targetAccept': .4, 'stepAdapt': .1}
    a = adaptation(s)
    assert a['STEP_MIN'] == .001 and a['STEP_MAX'] == .25
    assert abs(a['STEP_UP'] - math.exp(.06)) < 1e-9 and abs(a['STEP_DOWN'] - math.exp(-.04)) < 1e-9
    for change in ({'stepMin': 0}, {'stepMax': .0001}, {'stepInit': 1}, {'targetAccept': 0}, {'targetAccept': 1},
                   {'stepAdapt': -1}, {'stepAdapt': 1e9}, {'stepMin': float('nan')}):
        with pytest.raises(ValueError, match='adaptation'):
            adaptation(dict(s, **change))


def test_ladders_and_schedule():
    assign = np.array([0] * 19 + [1] * 8, dtype=np.uint32)
    lad, temp = build_ladders(assign, 8, 5e-4, 0.05)
    lad = lad.reshape(-1, 8)
    # assignment 0: two full ladders + three cold singletons; assignment 1: one ladder
    assert lad.shape[0] == 2 + 3 + 1
    assert list(lad[0]) == list(range(8)) and list(lad[1]) == list(range(8, 16))
    assert list(lad[2]) == [16] + [-1] * 7
    ratio = (0.05 / 5e-4) ** (1 / 7)
    assert np.allclose(temp[:8], [5e-4 * ratio ** r for r in range(8)], rtol=1e-6)
    assert temp[17] == np.float32(5e-4)
    g, p = schedule(5000, 87)
    assert g[0] == 22 and g[-1] == 87 and p[0] == np.float32(0.2) and p[-1] == np.float32(4.0)
    assert np.all(np.diff(g) >= 0) and len(set(g.tolist())) <= 24


def test_batched_problem_generator():
    """Uneven batch: the six space groups, 1-24 sites, at most 512 atoms per cell,
    replicas 256-2048 in multiples of 8, points 2000-12000."""
    from powder6_b200.workloads import BATCH_GROUPS, batched_problems
    items = batched_problems(12, seed=4)
    assert len(items) == 12
    for it in items:
        P = it.problem
        assert P.group.number in BATCH_GROUPS
        assert 1 <= P.max_sites <= 24
        assert sum(d['count'] for d in P.demand) <= 512
        assert 256 <= it.replicas <= 2048 and it.replicas % 8 == 0
        assert 2000 <= it.points <= 12000
        assert 8 <= P.refl.n_refl <= 3000
