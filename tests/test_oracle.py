"""The oracle itself: known answers and identities it must satisfy before the
kernels are compared against it."""
import ctypes as C
import math

import numpy as np
import pytest

from powder6_b200.swarm_wyckoff import cpu_cross_check


def test_philox_known_answers(oracle):
    lib = oracle.load()
    lib.p6o_philox.argtypes = [C.c_void_p] * 3
    for ctr, key, exp in [([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
                          ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
                          ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
                           [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1])]:
        c = np.array(ctr, dtype=np.uint32)
        k = np.array(key, dtype=np.uint32)
        o = np.zeros(4, dtype=np.uint32)
        lib.p6o_philox(c.ctypes.data, k.ctypes.data, o.ctypes.data)
        assert list(o) == exp


def _fit(O, P, coords, n_groups=None, refl=None, centro=None):
    ms = P.max_sites
    refl = refl or P.refl
    return O.wy_fitness(coords, P.tables.site_proj[:ms * 12], P.tables.gen_pack[:P.n_tot], P.sym_packed,
                        refl.group_meta, refl.n_groups if n_groups is None else n_groups, 4, refl.refl_pack,
                        P.f_tab, P.n_elem, P.centro if centro is None else centro)


def test_fitness_matches_product_cross_check_and_true_structure_scores_high(oracle, pbso4):
    cc, sums = _fit(oracle, pbso4, pbso4.true_coords)
    assert cc > 0.95
    assert abs(cc - cpu_cross_check(pbso4, pbso4.true_coords, 0)) < 1e-12
    # the sine terms cancel in a centrosymmetric cell
    cc2, _ = _fit(oracle, pbso4, pbso4.true_coords, centro=0)
    assert abs(cc - cc2) < 1e-12
    rnd = np.random.default_rng(7).random(pbso4.max_sites * 3)
    assert _fit(oracle, pbso4, rnd)[0] < 0.5


def test_wr2_identity_and_scale_freedom(oracle, pbso4):
    """wR2^2 = 1 - sco^2/(scc soo) (swarm_reflection.wgsl:237-257): an exact
    model scores 1 and an overall factor on Iobs changes nothing."""
    import copy
    P = pbso4
    x = P.true_coords
    # observations replaced by the model's own Icalc -> cc = 1
    ms = P.max_sites
    cc, (scc, soo, sco) = _fit(oracle, P, x)
    ic = _icalc_groups(P, x)
    R = copy.deepcopy(P.refl)
    gm = R.group_meta.reshape(-1, 4)
    gm[:, 2] = ic.astype(np.float32)
    assert _fit(oracle, P, x, refl=R)[0] > 1 - 1e-6
    gm[:, 2] *= 37.0
    assert _fit(oracle, P, x, refl=R)[0] > 1 - 1e-6
    # direct restatement of the identity
    wr2 = math.sqrt(max(0.0, 1 - sco * sco / (scc * soo)))
    assert abs(cc - (1 - wr2)) < 1e-12


def _icalc_groups(P, x):
    out = []
    # FP64 restatement through the product cross-check's arithmetic, per group
    import powder6_b200.swarm_wyckoff as sw
    T = P.tables
    ms = T.max_sites
    sp = T.site_proj[:ms * 12].astype(np.float64).reshape(ms, 12)
    proj = np.einsum('sij,sj->si', sp[:, :9].reshape(ms, 3, 3), np.asarray(x).reshape(ms, 3)) + sp[:, 9:]
    proj -= np.floor(proj)
    gp = T.gen_pack[:T.n_tot].astype(np.int64)
    site, op, ty = gp & 0xFF, (gp >> 8) & 0xFFF, (gp >> 20) & 0xF
    sym = P.sym_packed.astype(np.float64).reshape(-1, 12)
    g = np.einsum('aij,aj->ai', sym[op, :9].reshape(-1, 3, 3), proj[site]) + sym[op, 9:]
    pk = P.refl.refl_pack[0::2].astype(np.int64)
    hkl = np.stack([(pk & 0x3FF) - 512, ((pk >> 10) & 0x3FF) - 512, ((pk >> 20) & 0x3FF) - 512], 1)
    q = hkl @ g.T
    f = P.f_tab.astype(np.float64).reshape(-1, P.n_elem)[:, ty]
    F = (f * np.exp(2j * np.pi * q)).sum(1)
    ic = P.refl.refl_pack[1::2] * np.abs(F) ** 2
    gm = P.refl.group_meta.reshape(-1, 4)
    return np.array([ic[int(r[0]):int(r[0]) + int(r[1])].sum() for r in gm])


def test_fixed_point_orbit_matches_fp64_orbit(oracle, pbso4):
    P = pbso4
    ms = P.max_sites
    x = np.random.default_rng(11).random(ms * 3)
    sp = P.tables.site_proj[:ms * 12].astype(np.float64).reshape(ms, 12)
    proj = (np.einsum('sij,sj->si', sp[:, :9].reshape(ms, 3, 3), x.reshape(ms, 3)) + sp[:, 9:]) % 1.0
    X = np.floor(proj.reshape(-1) * 2 ** 32 + 0.5).astype(np.uint64).astype(np.uint32)
    rint = np.array([o.r for o in P.group.ops], dtype=np.int32).reshape(-1)
    tfix = np.array([[(t * 2 ** 32 + 12) // 24 for t in o.t] for o in P.group.ops], dtype=np.uint64).astype(np.uint32)
    fx = oracle.expand_fixed(X, P.tables.gen_pack[:P.n_tot], rint, tfix.reshape(-1)).reshape(-1, 3)
    gp = P.tables.gen_pack[:P.n_tot].astype(np.int64)
    site, op = gp & 0xFF, (gp >> 8) & 0xFFF
    sym = P.sym_packed.astype(np.float64).reshape(-1, 12)
    g = (np.einsum('aij,aj->ai', sym[op, :9].reshape(-1, 3, 3), (X.astype(np.float64) / 2 ** 32).reshape(ms, 3)[site])
         + sym[op, 9:]) % 1.0
    d = np.abs(fx.astype(np.float64) / 2 ** 32 - g)
    assert np.all(np.minimum(d, 1 - d) < 2 ** -30)


def test_acceptance_rule(oracle):
    su, sd, smin, smax = math.exp(0.056), math.exp(-0.024), 2e-4, 0.5
    # first evaluation of a chain: fit = -1e30 sentinel, always accepted, becomes best
    st = np.array([-1e30, float('nan'), 0, 0.08, 0.01, -1e30, 0, 0])
    acc, st2, best = oracle.wy_accept(st, 0.5, 0.1, 2.0, 0.99, su, sd, smin, smax)
    assert acc == 1 and best == 1 and abs(st2[0] - 0.4) < 1e-12 and abs(st2[2] - 0.05) < 1e-12
    assert abs(st2[3] - 0.08 * su) < 1e-12
    # incumbent re-scored at the current penScale: cc .6, raw pen .1 at scale 3 -> f_old .3
    st = np.array([0.55, 0.6, 0.1, 0.08, 0.01, 0.5, 0.6, 0.1])
    f_new = 0.6 - 0.32                                   # cc .6, pen .32 (scaled)
    p = math.exp((f_new - 0.3) / 0.01)
    assert oracle.wy_accept(st, 0.6, 0.32, 3.0, p * 0.999, su, sd, smin, smax)[0] == 1
    assert oracle.wy_accept(st, 0.6, 0.32, 3.0, p * 1.001, su, sd, smin, smax)[0] == 0
    rej = oracle.wy_accept(st, 0.6, 0.32, 3.0, 0.9999, su, sd, smin, smax)[1]
    assert abs(rej[3] - 0.08 * sd) < 1e-12 and rej[0] == 0.55
    # step clamped to its bounds
    st = np.array([0.5, 0.5, 0, 0.5, 0.01, -1e30, 0, 0])
    assert oracle.wy_accept(st, 0.9, 0, 1, 0.5, su, sd, smin, smax)[1][3] == 0.5


def test_penalty_clash_closed_form(oracle, pbso4):
    """Two atoms at a known separation below the floor: penClash (1 + 9 overlap)."""
    from powder6_b200.symmetry import space_group
    from powder6_b200.wyckoff_tables import build_assignment_tables, build_restraint_tables, make_assignment, pack_sym_ops
    from powder6_b200.crystal import reduced_cell
    g = space_group(1)
    cell = {'a': 10, 'b': 10, 'c': 10, 'alpha': 90, 'beta': 90, 'gamma': 90}
    demand = [{'element': 'C', 'count': 2, 'z': 6}]
    A = make_assignment(g, demand, [('C', '1a'), ('C', '1a')])
    T = build_assignment_tables([A], g, demand)
    R = build_restraint_tables(demand, [], min_contact=1.2)
    red = reduced_cell(cell)
    geom = oracle.make_geom(red.orth, red.xform, 0, 1, 0.05, 0.1, 0.03, 1.0, 2.0)
    proj = np.array([0.1, 0.1, 0.1, 0.18, 0.1, 0.1])              # 0.8 A apart
    pen = oracle.wy_penalty(proj, T.gen_pack, pack_sym_ops(g.ops), 1, R.tables, R.r_min_off, R.rule_off, 0, 64, 1, geom)
    # rMin is a float32 table, as in the reference
    assert abs(pen - 2.0 * 0.05 * (1 + 9 * (1.2 - 0.8) / 1.2)) < 1e-6
    proj = np.array([0.1, 0.1, 0.1, 0.95, 0.1, 0.1])              # 1.5 A through the cell face
    assert oracle.wy_penalty(proj, T.gen_pack, pack_sym_ops(g.ops), 1, R.tables, R.r_min_off, R.rule_off, 0, 64, 1, geom) == 0


def test_mlp_oracle_gradient_is_the_loss_derivative(oracle):
    """The FP64 network oracle's gradient against central differences of its loss."""
    rng = np.random.default_rng(2)
    d_in, width, d_out = 5, 7, 2
    n_par = d_in * width + width + width * width + width + width * d_out + d_out
    w = rng.normal(size=n_par) * 0.5
    X = rng.normal(size=(9, d_in))
    T = rng.normal(size=(9, d_out))
    M = (rng.random((9, d_out)) < 0.6).astype(float)
    g, loss = oracle.mlp_grads_fp64(w, X, T, M, d_in, width, d_out)
    for i in rng.choice(n_par, 12, replace=False):
        e = np.zeros(n_par)
        e[i] = 1e-6
        lp = oracle.mlp_grads_fp64(w + e, X, T, M, d_in, width, d_out)[1]
        lm = oracle.mlp_grads_fp64(w - e, X, T, M, d_in, width, d_out)[1]
        assert abs((lp - lm) / 2e-6 - g[i]) <= 1e-6 * max(1.0, abs(g[i]))
