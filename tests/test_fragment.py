"""The rigid-fragment parametrisation on the host: the config-5 molecule
(cimetidine's 17 non-H atoms from the reference's test file), its torsion
sets, and the product's parameter -> coordinate map against the oracle's FP64
restatement; bond lengths and angles hold under any parameters."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from powder6_b200.crystal import orth_matrix
from powder6_b200.fragment import (CIMETIDINE_TORSIONS, build_fragment, fragment_coords, fragment_problem,
                                   load_molecule, random_params)

CELL = {'a': 10.2, 'b': 12.1, 'c': 15.3, 'alpha': 90.0, 'beta': 100.0, 'gamma': 90.0}


@pytest.fixture(scope='module')
def frag():
    el, xyz, bonds = load_molecule()
    return build_fragment(el, xyz, bonds, CIMETIDINE_TORSIONS, CELL)


def test_molecule_and_torsions(frag):
    assert frag.n_atoms == 17
    assert sorted(set(frag.elements)) == ['C', 'N', 'S'] and frag.elements.count('C') == 10 \
        and frag.elements.count('N') == 6
    assert len(frag.bonds) == 17                       # 16 tree bonds + the imidazole ring closure
    # each torsion turns the side of its bond away from atom 0, axis atom b fixed, c turned
    for (b, c), m in zip(frag.torsions, frag.moving):
        assert (m >> c) & 1 and not (m >> b) & 1 and not m & 1
    # the chain from the guanidine to the ring: each torsion turns fewer atoms than the one before
    counts = [bin(m).count('1') for m in frag.moving]
    assert counts == sorted(counts, reverse=True) and counts[0] == 11


def test_map_matches_the_oracle_and_keeps_the_geometry(frag):
    orth = orth_matrix(CELL).astype(np.float64).reshape(3, 3)
    prm = random_params(np.random.default_rng(4), 20, len(frag.torsions))
    ref_d = {}
    for u, v in frag.bonds:
        ref_d[(u, v)] = np.linalg.norm(frag.ref[u] - frag.ref[v])
    for p in prm:
        mine = fragment_coords(frag, p)
        want = O.fragment_coords_fp64(frag.ref, [t[0] for t in frag.torsions], [t[1] for t in frag.torsions],
                                      frag.moving, frag.to_frac, p)
        d = mine - want
        d -= np.round(d)
        assert np.max(np.abs(d)) < 1e-12
        for (u, v), r0 in ref_d.items():
            e = mine[u] - mine[v]
            e -= np.round(e)
            assert abs(np.linalg.norm(orth @ e) - r0) < 1e-9
    # zero torsions and the identity orientation: the reference geometry shifted by t
    p = np.zeros(16)
    p[3] = 1.0
    p[:3] = [0.3, 0.4, 0.5]
    f = fragment_coords(frag, p)
    cart = (f - p[:3]) - np.round(f - p[:3] - (frag.ref @ frag.to_frac.T))
    assert np.allclose(cart @ orth.T, frag.ref, atol=1e-9)


def test_config5_problem():
    P, frag, truth = fragment_problem(seed=1)
    assert P.max_sites == 17 and P.n_tot == 68 and len(P.assignments) == 1
    assert 500 < P.refl.n_refl < 700
    # the true coordinates are the fragment at the true parameters
    assert np.allclose(P.true_coords[:51].reshape(17, 3), fragment_coords(frag, truth), atol=1e-12)
