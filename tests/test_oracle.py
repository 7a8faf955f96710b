"""CPU tests: the oracle against the reference's own known answers, and its internal laws.

The known answers come from the reference's GoogleTest suite (test/toy_example.hpp,
test/entropy_test.cpp, test/blockmodel_test.cpp, test/common_test.cpp, test/finetune_test.cpp,
test/block_merge_test.cpp), extracted into tests/golden/toy_example.json.  The reference
compares with EXPECT_FLOAT_EQ (FP32 logs); the oracle computes in FP64, so values that the
reference pins to FP32 are compared at 1e-6 relative.
"""
import numpy as np
import pytest

from conftest import random_assignment, random_graph, toy_fixture

FP32_REL = 1e-6


def toy(O, which="assignment", B=3):
    fx = toy_fixture()
    e = np.array(fx["edges"], np.int32)
    g = O.Graph(fx["num_vertices"], e[:, 0], e[:, 1])
    return fx, g, O.Blockmodel(g, B, np.array(fx[which], np.int32))


def test_philox_known_answers(O):
    # Random123 philox4x32-10 known-answer vectors
    assert list(O.philox([0, 0, 0, 0], [0, 0])) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert list(O.philox([0xffffffff] * 4, [0xffffffff] * 2)) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert list(O.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0])) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_toy_graph_shape(O):   # EntropyTest.SetUpWorksCorrectly
    fx, g, B = toy(O)
    assert g.V == 11 and g.E == 23


def test_toy_mdl_known_answer(O):   # EntropyTest.MDLGivesCorrectAnswer
    fx, g, B = toy(O)
    assert B.mdl() == pytest.approx(fx["mdl"], rel=FP32_REL)


def test_toy_block_degrees(O):   # BlockmodelTest.BlockDegreesAreCorrectlyInstantiated
    fx, g, B = toy(O)
    do, di, d = B.degrees()
    for k, v in fx["degrees"].items():
        name, blk = k[:-3], int(k[-2])
        arr = {"degrees_out": do, "degrees_in": di, "degrees": d}[name]
        assert arr[blk] == v, k


def test_null_mdl_known_answers(O):   # EntropyTest.NullModelMDL*
    fx = toy_fixture()
    assert O.null_mdl_v1(50) == pytest.approx(fx["null_mdl_v1_E50"], rel=FP32_REL)
    assert O.null_mdl_v2(10, 50) == pytest.approx(fx["null_mdl_v2_V10_E50"], rel=FP32_REL)
    assert O.null_mdl_v1(int(5e12)) == pytest.approx(1.462023e14, rel=1e-6)
    assert O.null_mdl_v2(int(1e12), int(5e12)) == pytest.approx(3.089407e14, rel=1e-6)


def test_toy_delta_mdl_equals_mdl_difference(O):   # EntropyTest.DeltaMDLUsingBlockmodelDeltasGivesCorrectAnswer
    fx, g, B = toy(O)
    before = B.mdl()
    dS, _ = B.delta_mdl_move(7, 0)
    B2 = B.copy()
    B2.move_vertex(7, 0)
    assert B2.matrix().sum() == g.E
    assert dS == pytest.approx(B2.mdl() - before, rel=1e-12)


def test_toy_move_matrix_delta(O):   # FinetuneTest.BlockmodelDeltasAreCorrect
    fx, g, B = toy(O)
    M0 = B.matrix()
    B2 = B.copy()
    B2.move_vertex(7, 0)
    diff = B2.matrix() - M0
    for k, v in fx["delta_move_7_to_0_with_self_in"].items():
        r, c = map(int, k.split(","))
        assert diff[r, c] == v, k
    # the move must equal a rebuild from the new assignment
    a = B.assignment()
    a[7] = 0
    assert np.array_equal(B2.matrix(), O.Blockmodel(g, 3, a).matrix())


def test_complex_move_delta_and_degrees(O):   # FinetuneTest.SpecialCaseBlockmodelDeltasAreCorrect
    fx, g, B = toy(O, "complex_assignment", 6)
    M0 = B.matrix()
    B2 = B.copy()
    B2.move_vertex(6, 0)
    diff = B2.matrix() - M0
    for k, v in fx["delta_complex_move_6_from_3_to_0"].items():
        r, c = map(int, k.split(","))
        assert diff[r, c] == v, k
    do, di, d = B2.degrees()
    exp = fx["complex_move_6_to_0_degrees"]
    assert list(do) == exp["out"] and list(di) == exp["in"]
    # Blockmodel::move_vertex(vertex, delta, proposal) sets d[3] from the already-updated
    # diagonal plus the delta; compute_new_block_degrees (the fixture) does not: they differ
    # exactly at the source block of the move.
    assert list(d) == [11, 7, 4, 7, 5, 6]
    assert exp["total_compute_new_block_degrees"][3] == 6
    dS, _ = B.delta_mdl_move(6, 0)
    assert dS == pytest.approx(B2.mdl() - B.mdl(), rel=1e-12)   # EntropyTest.SpecialCaseShouldGiveCorrectDeltaMDL


def test_toy_merge_delta_and_mdl(O):   # BlockMergeTest / BlockMergeEntropyTest
    fx, g, B = toy(O)
    am = np.array([1, 1, 1, 1, 1, 1, 1, 2, 2, 2, 2], np.int32)
    Bm = O.Blockmodel(g, 3, am)
    diff = Bm.matrix() - B.matrix()
    for k, v in fx["delta_merge_0_into_1"].items():
        r, c = map(int, k.split(","))
        assert diff[r, c] == v, k
    assert B.merge_delta_mdl(0, 1) == pytest.approx(Bm.mdl() - B.mdl(), rel=1e-12)


def quirk_term(edges, a, M, do, di, v, r, s):
    """Extra term the reference's delta_mdl adds for a present, net-zero (r,s)/(s,r) cell."""
    src, dst = edges
    out = dst[(src == v) & (dst != v)]
    inn = src[(dst == v) & (src != v)]
    co = np.bincount(a[out], minlength=len(do))
    ci = np.bincount(a[inn], minlength=len(do))
    k_out = int(((src == v)).sum())
    kin_self = int(len(inn) + ((src == v) & (dst == v)).sum())
    q = 0.0
    if (co[s] > 0 or ci[r] > 0) and ci[r] - co[s] == 0 and M[r, s] > 0:
        q += M[r, s] * (np.log((di[s] + kin_self) / di[s]) + np.log((do[r] - k_out) / do[r]))
    if (co[r] > 0 or ci[s] > 0) and co[r] - ci[s] == 0 and M[s, r] > 0:
        q += M[s, r] * (np.log((di[r] - kin_self) / di[r]) + np.log((do[s] + k_out) / do[s]))
    return q


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_delta_mdl_equals_mdl_difference_plus_quirk(O, seed):
    """delta_mdl == MDL(after) - MDL(before), plus the reference's double count of a present
    net-zero (r,s)/(s,r) Delta cell (src/entropy.cpp:344-371) when that case occurs."""
    V, s, d, _ = random_graph(150, 5, seed)
    g = O.Graph(V, s, d)
    pairs = np.unique(np.stack([s, d], 1), axis=0)
    edges = (pairs[:, 0], pairs[:, 1])
    rng = np.random.default_rng(seed)
    B = O.Blockmodel(g, 8, random_assignment(V, 8, seed))
    quirks = 0
    for _ in range(60):
        v = int(rng.integers(V))
        t = int(rng.integers(8))
        a = B.assignment()
        r = int(a[v])
        if t == r:
            continue
        a2 = a.copy()
        a2[v] = t
        after = O.Blockmodel(g, 8, a2)
        dS, _ = B.delta_mdl_move(v, t)
        do, di, _ = B.degrees()
        q = quirk_term(edges, a, B.matrix(), do, di, v, r, t)
        quirks += q != 0.0
        assert dS == pytest.approx(after.mdl() - B.mdl() + q, rel=1e-9, abs=1e-9)
        B.move_vertex(v, t)
        assert np.array_equal(B.matrix(), after.matrix())
    assert quirks > 0


def test_merge_delta_equals_mdl_difference_random(O):
    V, s, d, _ = random_graph(200, 6, 5)
    g = O.Graph(V, s, d)
    B = O.Blockmodel(g, 10, random_assignment(V, 10, 5))
    for r, t in [(0, 1), (3, 7), (9, 2), (5, 5 ^ 1)]:
        a = B.assignment()
        a[a == r] = t
        after = O.Blockmodel(g, 10, a)
        assert B.merge_delta_mdl(r, t) == pytest.approx(after.mdl() - B.mdl(), rel=1e-10)


@pytest.mark.parametrize("algo", [0, 1, 2])
def test_finetune_keeps_counts_consistent(O, algo):
    V, s, d, _ = random_graph(300, 6, 7)
    g = O.Graph(V, s, d)
    B = O.Blockmodel(g, 12, random_assignment(V, 12, 7))
    st = B.finetune(algo, batches=4, seed=3, max_sweeps=4)
    assert st["visits"] > 0 and st["accepted"] > 0
    rebuilt = O.Blockmodel(g, 12, B.assignment())
    assert np.array_equal(B.matrix(), rebuilt.matrix())
    do, di, _ = B.degrees()
    do2, di2, _ = rebuilt.degrees()
    assert np.array_equal(do, do2) and np.array_equal(di, di2)
    assert st["mdl"] == pytest.approx(rebuilt.mdl(), rel=1e-6)


def test_replay_records_equal_philox_stream(O):
    """A replay buffer holding the Philox records gives the same chain as the seeded run."""
    V, s, d, _ = random_graph(200, 5, 9)
    g = O.Graph(V, s, d)
    a = random_assignment(V, 10, 9)
    sweeps = 3
    rec = np.zeros((sweeps * V, 4), np.uint32)
    for sw in range(sweeps):
        for v in range(V):
            key = [0x1234, 0]
            rec[sw * V + v] = O.philox([v, sw, 0, 0], key)
    for algo in (0, 1):
        B1 = O.Blockmodel(g, 10, a)
        B2 = O.Blockmodel(g, 10, a)
        st1 = B1.finetune(algo, batches=3, seed=0x1234, max_sweeps=sweeps)
        st2 = B2.finetune(algo, batches=3, replay=rec, max_sweeps=sweeps)
        assert np.array_equal(B1.assignment(), B2.assignment())
        assert st1["accepted"] == st2["accepted"]


def test_sbp_small_recovers_planted_partition(O):
    V, s, d, truth = random_graph(400, 4, 13, kmin=8, kmax=40, w=0.9, alpha=10.0)
    g = O.Graph(V, s, d)
    out, st = O.sbp(g, algo=1, batches=4, seed=5)
    assert st["num_blocks"] >= 2
    assert O.nmi(out, truth) > 0.8
