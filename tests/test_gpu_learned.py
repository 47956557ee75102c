"""Proposal network and learned search.

Parity: the network's gradients (FP32 master weights) against the FP64
oracle within 1e-5 of the largest gradient; inference (bf16 weights and
activations on the tensor cores) within 5e-2 of the largest FP64 output
(bf16 carries ~3 significant digits at each of two hidden layers).  Gain:
trained on the plain search's own moves, ranking 8 candidates raises the
acceptance rate and the mean exact fitness change of the evaluated
proposals over the plain move, from the same search state."""
import numpy as np
import pytest

from powder6_b200.learned import (ProposalNet, collect_records, gain_targets, learned_problem, learned_step, start)
from powder6_b200.swarm_wyckoff import WyckoffSession

pytestmark = pytest.mark.gpu


def test_gradients_and_inference_match_oracle(oracle):
    rng = np.random.default_rng(0)
    X = rng.normal(size=(512, 64)).astype(np.float32)
    T = rng.normal(size=(512, 1)).astype(np.float32)
    M = (rng.random((512, 1)) < 0.7).astype(np.float32)
    with ProposalNet(64, 256, 1, seed=3) as net:
        w = net.params()
        for mask in (None, M):
            g, loss = net.gradients(X, T, mask)
            g64, l64 = oracle.mlp_grads_fp64(w, X, T, mask, 64, 256, 1)
            assert np.max(np.abs(g - g64)) <= 1e-5 * np.max(np.abs(g64))
            assert abs(loss - l64) <= 1e-5 * l64
        Y = net.predict(X)
        Y64 = oracle.mlp_forward_fp64(w, X, 64, 256, 1)[0]
        assert np.max(np.abs(Y - Y64)) <= 5e-2 * np.max(np.abs(Y64))
        # more rows than one tile, a partial last tile
        X3 = rng.normal(size=(1000, 64)).astype(np.float32)
        Y3 = net.predict(X3)
        Y3_64 = oracle.mlp_forward_fp64(w, X3, 64, 256, 1)[0]
        assert np.max(np.abs(Y3 - Y3_64)) <= 5e-2 * np.max(np.abs(Y3_64))


def test_training_fits_a_smooth_target():
    rng = np.random.default_rng(1)
    X = rng.normal(size=(2048, 64)).astype(np.float32)
    T = (np.sin(X[:, :1]) + X[:, 1:2] * X[:, 2:3]).astype(np.float32)
    with ProposalNet(64, 256, 1, seed=5) as net:
        losses = net.train(X, T, epochs=20, batch=256, lr=2e-3)
    assert losses[-1] < 0.05 * losses[0]


def test_learned_ranking_gains_over_the_plain_move():
    P = learned_problem()
    with WyckoffSession(P, 2048, run_key=5, incremental=0) as s:
        X, gains, acc = collect_records(s, P, 150, seed=4, every=2)
        T, _ = gain_targets(gains)
        with ProposalNet(64, 256, 1, seed=7) as net:
            net.train(X, T, epochs=4, batch=2048, lr=1e-3)
            X2, g2, _ = collect_records(s, P, 40, seed=9, every=4)
            corr = float(np.corrcoef(net.predict(X2)[:, 0], g2)[0, 1])
            groups, _ = start(s, P, 1000, seed=11)
            for g in range(200):
                learned_step(s, None, 1, g, g == 0 or groups[g] != groups[g - 1])
            cur, _, st = s.read_state()
            plain, learned = [], []
            for t in range(4):
                s.sync_state(cur, st)
                _, gp, ap, _ = learned_step(s, None, 1, 200 + t, True, records=True)
                s.sync_state(cur, st)
                _, gl, al, _ = learned_step(s, net, 8, 200 + t, True, records=True)
                plain.append((gp.mean(), ap.mean()))
                learned.append((gl.mean(), al.mean()))
    assert corr > 0.2
    plain, learned = np.array(plain), np.array(learned)
    assert learned[:, 0].mean() > plain[:, 0].mean()          # mean exact fitness change
    assert learned[:, 1].mean() > plain[:, 1].mean()          # acceptance
