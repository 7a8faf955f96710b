"""CPU checks of the learned-proposal oracle (oracle/learned_oracle.py) itself."""
import numpy as np
import pytest

from conftest import random_assignment, random_graph
import learned_oracle as LO


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-9, 3.14159, -2.5e-3, 65504.0], np.float32)
    got = LO.bf16(x)
    # ties go to even: 1 + 2^-8 is halfway between 1 and 1 + 2^-7
    assert got.tolist() == [1.0, 1.0, 1.0078125, 3.140625, float(np.float32(-0.0025024414)), 65536.0]


def test_exact_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, LO.PARAMS)
    X = rng.random((40, 64))
    nv = rng.integers(0, 15, 40)
    t = np.array([rng.integers(0, n) if n > 0 and rng.random() < 0.8 else LO.ESCAPE for n in nv])
    t[3] = -1
    g, loss = LO.gradients(p, X, t, nv, rounding=False)
    assert loss == pytest.approx(LO.loss_of(p, X, t, nv, rounding=False), rel=1e-12)
    h = 1e-6
    for i in rng.choice(LO.PARAMS, 80, replace=False):
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (LO.loss_of(pp, X, t, nv, rounding=False) - LO.loss_of(pm, X, t, nv, rounding=False)) / (2 * h)
        assert g[i] == pytest.approx(fd, rel=1e-5, abs=1e-8), i


def test_rounded_gradients_close_to_exact():
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.1, LO.PARAMS).astype(np.float32)
    X = rng.random((256, 64)).astype(np.float32)
    nv = rng.integers(1, 15, 256)
    t = np.array([rng.integers(0, n) for n in nv])
    g, _ = LO.gradients(p, X, t, nv)
    ge, _ = LO.gradients(p.astype(np.float64), X, t, nv, rounding=False)
    assert np.dot(g, ge) / (np.linalg.norm(g) * np.linalg.norm(ge)) > 0.99


def test_reverse_features_equal_features_after_the_move():
    """The property the exact Hastings factor rests on: the reverse-state features built from
    the current state are the features the vertex has once the move is made."""
    V, s, d, _ = random_graph(300, 6, 7)
    g = LO.Graph(V, s, d)
    B = 12
    b = random_assignment(V, B, 7)
    d_out, d_in = LO.block_degrees(g, b, B)
    rng = np.random.default_rng(3)
    for v in rng.choice(V, 60, replace=False):
        F1, slots, r, k_out, k_in, self = LO.vertex_features(g, b, B, d_out, d_in, v)
        for tgt in {int(rng.integers(0, B)), slots[0][0] if slots else 0}:
            if tgt == r:
                continue
            F2 = LO.reverse_features(F1, slots, r, tgt, k_out, k_in, self, B, d_out, d_in, g.E)
            b2 = b.copy()
            b2[v] = tgt
            do2, di2 = LO.block_degrees(g, b2, B)
            Fa, slots_a, _, _, _, _ = LO.vertex_features(g, b2, B, do2, di2, v)
            assert np.array_equal(F2.view(np.uint32), Fa.view(np.uint32))
            assert [x[0] for x in slots_a] == [x[0] for x in slots]


def test_mixture_probabilities_sum_to_one():
    rng = np.random.default_rng(5)
    B = 9
    for _ in range(20):
        L = rng.normal(0, 2, 16).astype(np.float32)
        nvalid = int(rng.integers(0, 10))
        slots = [(int(x), 1, 0) for x in rng.choice(B, nvalid, replace=False)]
        q = np.zeros(B)
        for blk in range(B):
            slot = next((j for j, x in enumerate(slots) if x[0] == blk), -1)
            q[blk] = LO.q_of(L, nvalid, slot, 0.05, B)
        assert q.sum() == pytest.approx(1.0, rel=1e-12)
        assert (q >= 0.05 / B).all()
