"""The Wyckoff worker's message protocol (js/wyckoff_worker.js:1782-1861) on
the host: job parsing, the message sequence and its fields, cancel between
launches and the answers to bad jobs.  The device search is replaced by a
stand-in with the same call signature, so these run on the CPU; the GPU test
in tests/test_gpu_wyckoff.py runs a job end to end on the device."""
import threading
import time

import numpy as np
import pytest

from powder6_b200.swarm_wyckoff import SearchResult
from powder6_b200.workloads import wyckoff_job, wyckoff_problem
from powder6_b200.wyckoff_worker import (WyckoffWorker, group_from_job, lorentz_polarisation, observation_rows,
                                         parse_formula, z_plan)

PROGRESS_FIELDS = {'type', 'wave', 'waves', 'generation', 'generations', 'restart', 'restarts', 'best', 'cc',
                   'assignment', 'bestSites', 'stage', 'fraction', 'z', 'zIndex', 'zCount'}


@pytest.fixture(scope='module')
def problem():
    return wyckoff_problem(seed=3)


def fake_search(delay=0.0, steps=5):
    calls = []

    def search(problem, n, generations, restarts, seed, settings=None, on_progress=None, should_stop=None,
               refine=True, chunk=None):
        calls.append({'n': n, 'generations': generations, 'restarts': restarts, 'seed': seed, 'chunk': chunk,
                      'n_assign': len(problem.assignments)})
        coords = np.full(problem.max_sites * 3, 0.137)
        for g in range(steps):
            if should_stop and should_stop():
                break
            on_progress({'restart': 1, 'restarts': restarts, 'generation': (g + 1) * generations // steps,
                         'generations': generations, 'fraction': (g + 1) / steps, 'best': 0.5, 'cc': 0.6,
                         'assignment': 0, 'coords': coords, 'wave': 1, 'waves': 1, 'stage': 'search'})
            time.sleep(delay)
        res = SearchResult(0.6, 0.01, coords, n * generations, 1.0, 0.5, float('nan'), 1, seed)
        res.best_assignment = 0
        res.per_assignment = {0: 0.6}
        res.refined = {0: {'coords': coords + 0.001, 'r_start': 0.4, 'r': 0.2, 'converged': True}}
        return res
    search.calls = calls
    return search


def run_job(job, search):
    out = []
    w = WyckoffWorker(out.append, search=search, threaded=False)
    w.on_message(job)
    return out


def test_formula_and_lp():
    assert parse_formula('PbSO4') == [('Pb', 1), ('S', 1), ('O', 4)]
    assert parse_formula('C10N6S') == [('C', 10), ('N', 6), ('S', 1)]
    assert parse_formula('Ca(OH)2') == [('Ca', 1), ('O', 2), ('H', 2)]
    # js/crystal.js:465-478: L = 1/(sin^2 th cos th), P = (1 + K cos^2 2th)/(1 + K)
    th = np.radians(20.0)
    assert lorentz_polarisation(40.0, 0.8) == pytest.approx(1 / (np.sin(th) ** 2 * np.cos(th)) *
                                                            (1 + 0.8 * np.cos(2 * th) ** 2) / 1.8, rel=1e-14)
    assert lorentz_polarisation(0.0, 1.0) == 1.0


def test_job_rebuilds_the_group_and_the_observations(problem):
    job = wyckoff_job(problem)
    g = group_from_job(job['symops'], job['wyckoffTable'])
    assert sorted((o.r, o.t) for o in g.ops) == sorted((o.r, o.t) for o in problem.group.ops)
    for a, b in zip(g.wyckoff, problem.group.wyckoff):
        assert (a.letter, a.multiplicity, a.P, a.T, a.coset_ops) == (b.letter, b.multiplicity, b.P, b.T, b.coset_ops)
    # the same operators as x,y,z strings
    xyz = []
    for o in problem.group.ops:
        comps = []
        for i in range(3):
            terms = ''.join(('+' if o.r[3 * i + k] > 0 else '-') + 'xyz'[k] for k in range(3) if o.r[3 * i + k])
            if o.t[i]:
                terms += f'+{o.t[i]}/24'
            comps.append(terms.lstrip('+'))
        xyz.append({'xyz': ','.join(comps)})
    g2 = group_from_job(xyz, job['wyckoffTable'])
    assert sorted((o.r, o.t) for o in g2.ops) == sorted((o.r, o.t) for o in g.ops)
    rows, warn = observation_rows(job)
    assert not warn and len(rows) == len(problem.rows)
    want = {(r['h'], r['k'], r['l']): r for r in problem.rows}
    for r in rows:
        w = want[(r['h'], r['k'], r['l'])]
        assert r['Fo2'] == pytest.approx(w['Fo2'], rel=1e-12)
        assert r['sigma'] == pytest.approx(w['sigma'], rel=1e-12)
    # without the per-row Lp the same values come from 2-theta and K
    for p in job['hklList']:
        p.pop('lp')
    rows2, _ = observation_rows(job)
    assert [r['Fo2'] for r in rows2] == pytest.approx([r['Fo2'] for r in rows], rel=1e-12)
    # negatives and non-numbers are dropped and counted
    job['hklList'][0]['intensity'] = -1.0
    job['hklList'][1]['intensity'] = 'n/a'
    rows3, warn3 = observation_rows(job)
    assert len(rows3) == len(rows) - 2 and 'NEGATIVE' in warn3[0] and '1 non-numeric' in warn3[0]


def test_message_sequence_and_fields(problem):
    search = fake_search()
    msgs = run_job(wyckoff_job(problem, swarmParticles=1000, swarmIterations=200, swarmRestarts=2), search)
    kinds = [m['type'] for m in msgs]
    assert kinds[0] == 'wy-start' and kinds[-1] == 'wy-structure'
    assert kinds.count('wy-progress') == 5 and kinds.count('wy-partial') == 1
    assert 'wy-error' not in kinds
    for m in msgs:
        if m['type'] == 'wy-progress':
            assert set(m) == PROGRESS_FIELDS
            assert m['z'] == 4 and m['zIndex'] == 1 and m['zCount'] == 1
            assert sum(x['multiplicity'] for x in m['bestSites']) == 24   # Pb4 S4 O16
    c = search.calls[0]
    # particles rounded up to whole ladders of 8; the enumeration found PbSO4's assignments
    assert (c['n'], c['generations'], c['restarts'], c['seed']) == (1000, 200, 2, 1)
    assert c['n_assign'] > 1
    res = msgs[-1]['results']
    assert res['source'] == 'wyckoff' and res['z'] == 4 and not res['stopped'] and not res['autoZ']
    assert res['refinement'] == {'R': 0.2, 'RStart': 0.4, 'converged': True}
    assert res['map'] is None and res['nOps'] == len(problem.group.ops)
    sites = res['sites']
    assert sum(s['multiplicity'] for s in sites) == 24
    for s in sites:
        assert set(s) == {'element', 'wyckoff', 'multiplicity', 'siteSymmetry', 'x', 'y', 'z'}
        assert all(0.0 <= s[a] < 1.0 for a in 'xyz')


def test_cancel_between_launches(problem):
    search = fake_search(delay=0.05, steps=50)
    out = []
    done = threading.Event()
    w = WyckoffWorker(None, search=search, threaded=True)

    def post(m):
        out.append(m)
        if m['type'] == 'wy-progress' and sum(1 for x in out if x['type'] == 'wy-progress') == 2:
            w.on_message({'type': 'cancel-wyckoff'})   # arrives while the search runs, gets no answer
        if m['type'] in ('wy-structure', 'wy-error'):
            done.set()
    w.post = post
    w.on_message(wyckoff_job(problem, swarmIterations=100))
    assert done.wait(30) and w.join(5)
    kinds = [m['type'] for m in out]
    assert kinds.count('wy-progress') == 2
    assert kinds[-1] == 'wy-structure' and out[-1]['results']['stopped']


def test_every_other_message_is_answered(problem):
    out = []
    w = WyckoffWorker(out.append, search=fake_search(), threaded=False)
    w.on_message({'type': 'charge-flip'})
    w.on_message(None)
    assert [m['type'] for m in out] == ['wy-error', 'wy-error']
    assert 'does not handle job type "charge-flip"' in out[0]['message']
    job = wyckoff_job(problem)
    for key, text in (('symops', 'No symmetry operators'), ('targetComposition', 'target composition'),
                      ('wyckoffTable', 'no Wyckoff table')):
        bad = dict(job)
        bad[key] = [] if key != 'targetComposition' else ''
        msgs = run_job(bad, fake_search())
        assert msgs[-1]['type'] == 'wy-error' and text in msgs[-1]['message']
    # a composition with no assignment at this Z is an error naming it
    msgs = run_job(dict(job, targetComposition='PbSO4', wyckoffZ=1), fake_search())
    assert msgs[-1]['type'] == 'wy-error' and 'Pb' in msgs[-1]['message']


def test_automatic_z_from_density(problem):
    job = wyckoff_job(problem)
    job.pop('wyckoffZ')
    g = group_from_job(job['symops'], job['wyckoffTable'])
    plan, auto = z_plan(dict(job, densityMin=5.0, densityMax=8.0), parse_formula('PbSO4'), g)
    # PbSO4: 303.26 g/mol in 318.7 A^3 -> Z = 4 at 6.32 g/cm^3
    assert auto and plan[0] == 4
    search = fake_search()
    msgs = run_job(dict(job, densityMin=2.0, densityMax=14.0, maxZSearches=3), search)
    res = msgs[-1]['results']
    assert msgs[-1]['type'] == 'wy-structure' and res['autoZ']
    # Z values with no assignment (odd Z in Pnma) are recorded, the others searched
    assert len(res['zPlan']) == 3 and res['z'] in res['zPlan']
    assert sum(1 for m in msgs if m['type'] == 'wy-partial') == len(search.calls)
