"""Wyckoff assignment enumeration against the reference's regression tests
(tests/regressions.test.cjs:571-578, :598-606) and the search's own
PbSO4 workload."""
import pytest

from powder6_b200.symmetry import space_group
from powder6_b200.wyckoff_assign import (coordination_compatible, dedupe_equivalent_assignments,
                                         enumerate_assignments, multisets_summing_to, normalizer_permutations,
                                         to_search_assignment)


def el(e, n, z):
    return {'element': e, 'count': n, 'z': z, 'r': 1}


def count(number, demand):
    g = space_group(number)
    en = enumerate_assignments(g, demand, {'ceiling': 24})
    return [len(en['assignments']), len(dedupe_equivalent_assignments(en['assignments'], g)['assignments'])]


def test_origin_shift_and_inversion_equivalents_are_searched_once():
    """tests/regressions.test.cjs:574-578: P4/mmm 1a, 1b, 1c, 1d are one
    placement; NaCl in P4/mmm has 12 assignments and 3 structures; Pb2O2 in
    P-1 has 477 assignments and 78 after the eight inversion centres are
    identified."""
    assert count(123, [el('NA', 1, 11)]) == [4, 1]
    assert count(123, [el('NA', 1, 11), el('CL', 1, 17)]) == [12, 3]
    assert count(2, [el('PB', 2, 82), el('O', 2, 8)]) == [477, 78]


def test_stated_geometry_rules_out_inversion_centres():
    """tests/regressions.test.cjs:605-606: in P-1 a square-planar Cu may sit
    on an inversion centre, a tetrahedral one may not (and the error names the
    coordination, not the caps)."""
    g = space_group(2)
    demand = [el('CU', 1, 29), el('O', 4, 8)]

    def run(geometry):
        return enumerate_assignments(g, demand, {'ceiling': 24,
                                                 'coordination': {'CU': {'count': 4, 'geometry': geometry}}})
    assert len(run('square-planar')['assignments']) > 0
    bad = run('tetrahedral')
    assert bad['assignments'] == [] and 'coordination stated for Cu' in bad['error']


def test_sulfur_is_kept_off_pnma_4a_and_the_workload_assignment_is_enumerated():
    """Pnma 4a has site symmetry -1: four-coordinate S (a tetrahedral former)
    cannot sit there, parity forbids odd coordination on it, and a site
    without inversion accepts anything.  PbSO4 (Z = 4) enumerates 35
    assignments, the search workload's Pb 4c, S 4c, O 4c, O 4c, O 8d among
    them, and it converts to the search's assignment type."""
    g = space_group(62)
    w4a, w4c = g.position('4a'), g.position('4c')
    ops = [(tuple(o.r), tuple(o.t_frac)) for o in g.ops]
    assert 'inversion centre' in coordination_compatible(w4a, 'S', {'count': 4}, ops)
    assert 'odd number' in coordination_compatible(w4a, 'NA', {'count': 3}, ops)
    assert coordination_compatible(w4c, 'S', {'count': 4}, ops) is None
    demand = [el('PB', 4, 82), el('S', 4, 16), el('O', 16, 8)]
    en = enumerate_assignments(g, demand, {'ceiling': 24})
    assert len(en['assignments']) == 35 and not en['truncated']
    labels = [sorted((s['element'], f"{g.wyckoff[s['wIdx']].multiplicity}{g.wyckoff[s['wIdx']].letter}")
                     for s in a['sites']) for a in en['assignments']]
    want = sorted([('PB', '4c'), ('S', '4c'), ('O', '4c'), ('O', '4c'), ('O', '8d')])
    assert want in labels
    a = to_search_assignment(g, en['assignments'][labels.index(want)])
    assert sum(s.w.multiplicity for s in a.sites) == 24
    with_s = enumerate_assignments(g, demand, {'ceiling': 24, 'coordination': {'S': {'count': 4}}})
    assert all(not (s['element'] == 'S' and g.wyckoff[s['wIdx']].letter in 'ab')
               for a in with_s['assignments'] for s in a['sites'])


def test_multisets_and_failure_messages():
    """Fixed points at most once, free positions up to maxRepeat; a count no
    multiplicity combination reaches, and elements competing for the same
    fixed points, are reported with their cause."""
    g = space_group(123)
    out = multisets_summing_to([g.position('1a'), g.position('1b'), g.position('2g')], 2,
                               {'maxSites': 4, 'maxRepeat': 4, 'maxPerElement': 500})
    assert sorted(map(sorted, out)) == [[0, 1], [2]]
    bad = enumerate_assignments(space_group(225), [el('NA', 3, 11)], {'ceiling': 24})
    assert bad['assignments'] == [] and 'common factor' in bad['error']
    clash = enumerate_assignments(g, [el('A', 1, 20), el('B', 1, 30), el('C', 1, 40), el('D', 1, 50),
                                      el('E', 1, 60)], {'ceiling': 24})
    assert clash['assignments'] == [] and 'fixed point holds one element' in clash['error']
    assert len(normalizer_permutations(space_group(1))) == 0


def enumerated_pbso4_alternatives():
    """The deduplicated PbSO4 assignments in Pnma with tetrahedral S, the
    search workload's own (true) assignment removed: the extra assignments a
    search over the enumeration gets."""
    from powder6_b200.wyckoff_assign import assignment_labels
    g = space_group(62)
    demand = [el('PB', 4, 82), el('S', 4, 16), el('O', 16, 8)]
    en = enumerate_assignments(g, demand, {'ceiling': 24, 'coordination': {'S': {'count': 4}}})
    kept = dedupe_equivalent_assignments(en['assignments'], g)['assignments']
    labels = [assignment_labels(g, a) for a in kept]
    true = sorted([('PB', '4c'), ('S', '4c'), ('O', '4c'), ('O', '4c'), ('O', '8d')])
    return [lab for lab in labels if sorted(lab) != true], len(labels)


def test_enumerated_assignments_build_search_tables():
    """Twelve assignments survive the coordination filter and deduplication;
    the eleven besides the true one build the search's packed tables next to
    it (every assignment generates the same 24 atoms per cell)."""
    from powder6_b200.workloads import wyckoff_problem
    alts, n = enumerated_pbso4_alternatives()
    assert n == 12 and len(alts) == 11
    P = wyckoff_problem(seed=1, extra_assignments=alts)
    assert len(P.assignments) == 12 and P.n_tot == 24
