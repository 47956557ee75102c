"""Reflection enumeration and observation packing.

The product enumeration (numpy) must equal the FP64 C restatement of
generateReflections (js/rietveld_core.js:247-276) bit for bit: indices,
multiplicities, d-spacings and order."""
import ctypes as C
import math

import numpy as np
import pytest

from powder6_b200.reflections import (gaussian_form_factor, generate_reflections, pack_reflections,
                                      ramped_group_count, scattering_table, unpack_hkl)
from powder6_b200.symmetry import group_from_hall, space_group
from powder6_b200.workloads import load_form_factor_table

CASES = [
    (225, {'a': 5.64, 'b': 5.64, 'c': 5.64, 'alpha': 90, 'beta': 90, 'gamma': 90}, 0.85),
    (62, {'a': 8.48, 'b': 5.40, 'c': 6.96, 'alpha': 90, 'beta': 90, 'gamma': 90}, 1.2),
    (14, {'a': 10.2, 'b': 12.1, 'c': 15.3, 'alpha': 90, 'beta': 100, 'gamma': 90}, 1.5),
    (176, {'a': 9.4, 'b': 9.4, 'c': 6.9, 'alpha': 90, 'beta': 90, 'gamma': 120}, 1.1),
    (166, {'a': 4.9, 'b': 4.9, 'c': 13.9, 'alpha': 90, 'beta': 90, 'gamma': 120}, 0.9),
    (2, {'a': 4.9, 'b': 5.6, 'c': 6.1, 'alpha': 88, 'beta': 96, 'gamma': 91}, 1.3),
    (15, {'a': 9.7, 'b': 8.9, 'c': 5.3, 'alpha': 90, 'beta': 105.7, 'gamma': 90}, 1.25),
]


def oracle_reflections(O, cell, ops, dmin, box=None):
    lib = O.load()
    lib.p6o_generate_reflections.restype = C.c_int
    lib.p6o_generate_reflections.argtypes = [C.c_void_p] * 4 + [C.c_double] + [C.c_void_p] * 6 + [C.c_int]
    c6 = np.array([cell['a'], cell['b'], cell['c'], cell['alpha'], cell['beta'], cell['gamma']], dtype=np.float64)
    rot = np.array([o.r for o in ops], dtype=np.int32).reshape(-1)
    tr = np.array([o.t_frac for o in ops], dtype=np.float64).reshape(-1)
    bx = None if box is None else np.array(box, dtype=np.int32)
    cap = 200000
    h, k, l, m = (np.zeros(cap, dtype=np.int32) for _ in range(4))
    d0 = np.zeros(cap)
    n = lib.p6o_generate_reflections(c6.ctypes.data, rot.ctypes.data, tr.ctypes.data, len(ops), dmin,
                                     None if bx is None else bx.ctypes.data, h.ctypes.data, k.ctypes.data,
                                     l.ctypes.data, m.ctypes.data, d0.ctypes.data, cap)
    return h[:n], k[:n], l[:n], m[:n], d0[:n]


@pytest.mark.parametrize('number,cell,dmin', CASES)
def test_enumeration_bit_exact_against_oracle(oracle, number, cell, dmin):
    g = space_group(number)
    mine = generate_reflections(cell, g.ops, dmin, with_eq=True)
    h, k, l, m, d0 = oracle_reflections(oracle, cell, g.ops, dmin)
    assert len(mine) == len(h) > 0
    assert [r.h for r in mine] == list(h)
    assert [r.k for r in mine] == list(k)
    assert [r.l for r in mine] == list(l)
    assert [r.m for r in mine] == list(m)
    assert np.array_equal(np.array([r.d0 for r in mine]).view(np.uint64), d0.view(np.uint64))
    assert all(len(r.eq) == r.m for r in mine)


def test_multiplicities_and_extinctions_closed_form():
    cell = {'a': 5.64, 'b': 5.64, 'c': 5.64, 'alpha': 90, 'beta': 90, 'gamma': 90}
    refl = {(r.h, r.k, r.l): r.m for r in generate_reflections(cell, space_group(225).ops, 0.85)}
    # F-centring: h, k, l all even or all odd; m-3m multiplicities
    assert all((h % 2 == k % 2 == l % 2) for (h, k, l) in refl)
    assert refl[(1, 1, 1)] == 8 and refl[(2, 0, 0)] == 6 and refl[(2, 2, 0)] == 12
    assert refl[(3, 1, 1)] == 24 and refl[(4, 2, 0)] == 24 and refl[(5, 3, 1)] == 48
    # Pnma: 0kl with k + l odd and hk0 with h odd are absent (n glide, a glide)
    cell2 = {'a': 8.48, 'b': 5.40, 'c': 6.96, 'alpha': 90, 'beta': 90, 'gamma': 90}
    r2 = {(r.h, r.k, r.l) for r in generate_reflections(cell2, space_group(62).ops, 1.2)}
    assert all(not (h == 0 and (k + l) % 2) for (h, k, l) in r2)
    assert all(not (l == 0 and h % 2) for (h, k, l) in r2)


def test_envelope_covers_expanded_and_oblique_cells():
    """regressions.test.cjs:1035-1042: the PT envelope of P1 covers trial cells."""
    ops = group_from_hall('P 1')
    initial = {'a': 3, 'b': 4, 'c': 5, 'alpha': 90, 'beta': 90, 'gamma': 90}
    keys = {(r.h, r.k, r.l) for r in generate_reflections(initial, ops, 1, box=[6, 8, 10], with_eq=False)}
    for cell in ({'a': 6, 'b': 8, 'c': 10, 'alpha': 90, 'beta': 90, 'gamma': 90},
                 {'a': 5, 'b': 7, 'c': 9, 'alpha': 72, 'beta': 108, 'gamma': 115}):
        for r in generate_reflections(cell, ops, 1, with_eq=False):
            assert (r.h, r.k, r.l) in keys


def _rows():
    return [
        {'h': 1, 'k': 0, 'l': 0, 'mult': 2, 'Fo2': 100.0, 'sigma': 10.0, 'd': 5.0},
        {'h': 0, 'k': 1, 'l': 0, 'mult': 2, 'Fo2': 50.0, 'sigma': 5.0, 'd': 5.005},   # within 0.2 % of d
        {'h': 1, 'k': 1, 'l': 0, 'mult': 4, 'Fo2': 30.0, 'sigma': 3.0, 'd': 3.5},
        {'h': -2, 'k': 1, 'l': 3, 'mult': 4, 'Fo2': 10.0, 'sigma': 0.0, 'd': 2.0},    # no sigma: dropped
    ]


def test_pack_reflections_groups_weights_and_bit_layout():
    P = pack_reflections(_rows())
    assert P.n_groups == 3 and P.n_refl == 4
    gm = P.group_meta.reshape(-1, 4)
    # sorted by d descending; the first two lines merge
    assert unpack_hkl(int(P.refl_pack[0])) == (0, 1, 0) and unpack_hkl(int(P.refl_pack[2])) == (1, 0, 0)
    assert gm[0, 0] == 0 and gm[0, 1] == 2 and gm[0, 2] == np.float32(2 * 50.0 + 2 * 100.0)
    assert unpack_hkl(int(P.refl_pack[6])) == (-2, 1, 3)
    assert gm[2, 3] == 0.0                                  # dropped, not unit weight
    w = [1 / ((2 * 5.0) ** 2 + (2 * 10.0) ** 2), 1 / (4 * 3.0) ** 2]
    mean = (np.float32(w[0]) + np.float32(w[1])) / 2
    assert abs(gm[0, 3] - np.float32(w[0]) / mean) < 1e-6 and abs(gm[1, 3] - np.float32(w[1]) / mean) < 1e-6
    assert abs(float(gm[:2, 3].mean()) - 1.0) < 1e-6         # normalised to mean 1


def test_pack_reflections_unweighted_and_range_check():
    rows = [dict(r, sigma=None) for r in _rows()]
    P = pack_reflections(rows)
    assert np.all(P.group_meta.reshape(-1, 4)[:, 3] == 1.0)
    with pytest.raises(ValueError, match='511'):
        pack_reflections([{'h': 600, 'k': 0, 'l': 0, 'mult': 2, 'Fo2': 1.0, 'sigma': 1.0, 'd': 1.0}])


def test_profile_width_grouping():
    rows = [{'h': i, 'k': 0, 'l': 0, 'mult': 2, 'Fo2': 1.0, 'sigma': 1.0, 'd': 5.0 / (1 + 0.01 * i), 'tth': 20 + 0.05 * i}
            for i in range(1, 6)]
    P = pack_reflections(rows, fwhm_at=lambda t: 0.2)       # lines 0.05 apart, half-width 0.1: one cluster
    assert P.n_groups == 1 and P.grouped_by == 'profile-width'
    P2 = pack_reflections(rows, fwhm_at=lambda t: 0.05)
    assert P2.n_groups == 5


def test_scattering_table_and_ramp():
    ff = gaussian_form_factor(load_form_factor_table())
    assert abs(ff('O', 0.0) - 8.0) < 0.25 and abs(ff('Pb', 0.0) - 82.0) < 0.3   # f(0) ~ Z
    P = pack_reflections(_rows())
    tab, ne, missing = scattering_table(P, [{'element': 'O', 'z': 8}, {'element': 'Xx', 'z': 3}], ff, 1.5)
    assert ne == 2 and missing == ['Xx']
    s = float(P.refl_s[0])
    dw = math.exp(-1.5 * s * s / 4)
    assert tab[0] == np.float32(ff('O', s) * dw) and tab[1] == np.float32(3 * dw)   # f = Z also takes the B factor
    # rampedGroupCount: at least 8, at most nGroups, linear from startFrac
    assert ramped_group_count(100, 0, 23) == 25
    assert ramped_group_count(100, 23, 23) == 100
    assert ramped_group_count(10, 0, 23) == 8
    assert ramped_group_count(100, 7, 23) == round(100 * (0.25 + 0.75 * 7 / (23 * 0.6)))
