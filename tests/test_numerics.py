"""Closed-form checks restated from the reference's tests/numerics.test.cjs:12-40
(cell volumes and d-spacings worked out by hand)."""
import math

import numpy as np

from powder6_b200.crystal import build_inv_dsq, cell_volume, inv_dsq, orth_matrix, reduced_cell


def d_spacing(cell, h, k, l):
    f = build_inv_dsq(cell)
    q = inv_dsq(f, h, k, l)
    return 1 / math.sqrt(q) if q > 0 else None


def near(a, b, tol):
    assert abs(a - b) <= tol, (a, b)


def test_cell_volumes_match_closed_forms():
    near(cell_volume({'a': 5, 'b': 5, 'c': 5, 'alpha': 90, 'beta': 90, 'gamma': 90}), 125, 1e-9)
    near(cell_volume({'a': 4, 'b': 4, 'c': 6, 'alpha': 90, 'beta': 90, 'gamma': 120}),
         16 * 6 * math.sin(math.pi * 2 / 3), 1e-9)
    near(cell_volume({'a': 5, 'b': 6, 'c': 7, 'alpha': 90, 'beta': 100, 'gamma': 90}),
         210 * math.sin(100 * math.pi / 180), 1e-9)
    near(cell_volume({'a': 5, 'b': 5, 'c': 5, 'alpha': 60, 'beta': 60, 'gamma': 60}), 125 / math.sqrt(2), 1e-9)


def test_d_spacings_match_closed_forms():
    cubic = {'a': 5, 'b': 5, 'c': 5, 'alpha': 90, 'beta': 90, 'gamma': 90}
    near(d_spacing(cubic, 1, 1, 1), 5 / math.sqrt(3), 1e-12)
    near(d_spacing(cubic, 2, 0, 0), 2.5, 1e-12)
    ortho = {'a': 5, 'b': 6, 'c': 7, 'alpha': 90, 'beta': 90, 'gamma': 90}
    near(d_spacing(ortho, 1, 2, 3), 1 / math.sqrt(1 / 25 + 4 / 36 + 9 / 49), 1e-12)
    hexa = {'a': 4, 'b': 4, 'c': 6, 'alpha': 90, 'beta': 90, 'gamma': 120}
    near(d_spacing(hexa, 1, 0, 0), 4 * math.sqrt(3) / 2, 1e-12)
    near(d_spacing(hexa, 0, 0, 1), 6, 1e-12)
    near(d_spacing(hexa, 1, 1, 0), 2, 1e-12)
    mono = {'a': 5, 'b': 6, 'c': 7, 'alpha': 90, 'beta': 100, 'gamma': 90}
    sb, cb = math.sin(100 * math.pi / 180), math.cos(100 * math.pi / 180)
    q = (1 / 25 + 4 / 49 - 2 * 2 * cb / 35) / (sb * sb) + 9 / 36
    near(d_spacing(mono, 1, 3, 2), 1 / math.sqrt(q), 1e-12)


def test_unusable_cell_gives_none():
    assert build_inv_dsq({'a': 5, 'b': 5, 'c': 5, 'alpha': 90, 'beta': 90, 'gamma': 0}) is None
    assert d_spacing({'a': 5, 'b': 5, 'c': 5, 'alpha': 90, 'beta': 90, 'gamma': 90}, 0, 0, 0) is None


def test_reduced_cell_is_the_same_lattice_and_rounding_is_safe():
    cell = {'a': 5, 'b': 6, 'c': 7, 'alpha': 80, 'beta': 120, 'gamma': 110}
    red = reduced_cell(cell)
    x = red.xform.reshape(3, 3)
    assert np.allclose(x, np.rint(x)) and abs(abs(np.linalg.det(x)) - 1) < 1e-9
    # a separation well inside the safe radius: independent rounding finds the nearest image
    o = orth_matrix(cell).astype(np.float64).reshape(3, 3)
    rng = np.random.default_rng(3)
    for _ in range(200):
        d = rng.random(3) - 0.5
        best = min(np.linalg.norm(o @ (d + np.array([i, j, k]))) for i in range(-3, 4)
                   for j in range(-3, 4) for k in range(-3, 4))
        q = x @ d
        q -= np.round(q)
        got = np.linalg.norm(red.orth.reshape(3, 3) @ q)
        if best < red.safe_radius:
            assert abs(got - best) < 1e-9
