"""Partition metrics (evaluate::calculate_f1_score / calculate_nmi / the Hungarian matching,
src/evaluate.cpp:7-178).

CPU: the oracle and the engine's host metrics (sbp_contingency_metrics) against the reference's
own known answers (test/evaluate_test.cpp, extracted into tests/golden/evaluate_known_answers.json),
and against each other on random tables, accuracy included (scipy's assignment solver on the
oracle side).
GPU: sbp_evaluate_blockmodel (contingency table counted on the device) against the oracle on
partitions of a benchmark-law graph, with and without unknown true labels.
"""
import json
import os

import numpy as np
import pytest

from conftest import ROOT, random_assignment, random_graph


def known():
    with open(os.path.join(ROOT, "tests", "golden", "evaluate_known_answers.json")) as f:
        return json.load(f)


def test_oracle_metrics_match_the_reference_known_answers(O):
    k = known()
    m = O.contingency_metrics(np.array(k["matrix"]), k["num_vertices"])
    # the reference's EXPECT_FLOAT_EQ values are printed to 6 significant digits
    for key in ("f1", "rand_index", "precision", "recall"):
        assert m[key] == pytest.approx(k[key], rel=2e-6), key
    m2 = O.contingency_metrics(np.array(k["matrix2"]), k["num_vertices2"])
    assert m2["f1"] == pytest.approx(k["f1_2"], rel=1e-7)


def test_engine_metrics_match_the_reference_known_answers():
    import sbp_b200 as S
    k = known()
    m = S.evaluate.contingency_metrics(np.array(k["matrix"]), k["num_vertices"])
    assert m["f1_score"] == pytest.approx(k["f1"], rel=2e-6)
    assert m["rand_index"] == pytest.approx(k["rand_index"], rel=2e-6)
    assert m["precision"] == pytest.approx(k["precision"], rel=2e-6)
    assert m["recall"] == pytest.approx(k["recall"], rel=2e-6)
    m2 = S.evaluate.contingency_metrics(np.array(k["matrix2"]), k["num_vertices2"])
    assert m2["f1_score"] == pytest.approx(k["f1_2"], rel=1e-7)


@pytest.mark.parametrize("shape,seed", [((5, 8), 1), ((8, 5), 2), ((30, 30), 3), ((64, 12), 4), ((1, 7), 5)])
def test_engine_metrics_match_the_oracle_on_random_tables(O, shape, seed):
    import sbp_b200 as S
    rng = np.random.default_rng(seed)
    t = rng.integers(0, 50, shape) * (rng.random(shape) < 0.4)
    t[0, 0] += 5
    N = int(t.sum())
    m, o = S.evaluate.contingency_metrics(t, N), O.contingency_metrics(t, N)
    assert m["accuracy"] == pytest.approx(o["accuracy"], rel=0, abs=0)
    for a, b in (("f1_score", "f1"), ("precision", "precision"), ("recall", "recall"), ("rand_index", "rand_index")):
        assert m[a] == pytest.approx(o[b], rel=1e-12), a
    if shape[0] > 1:
        assert m["nmi"] == pytest.approx(o["nmi"], rel=1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("unknown", [False, True])
def test_device_evaluation_matches_the_oracle(S, O, unknown):
    V, s, d, truth = random_graph(20000, 12, 31)
    g = S.Graph(V, s, d)
    truth = truth.astype(np.int32) * 7 + 3   # community ids that are not 0..K-1
    if unknown:
        truth[::11] = -1
    for B, seed in ((12, 1), (40, 2), (300, 3)):
        a = random_assignment(V, B, seed)
        a[: V // 2] = np.where(truth[: V // 2] >= 0, (truth[: V // 2] // 7) % B, a[: V // 2])
        bm = S.Blockmodel(g, B, a)
        ev = S.evaluate.evaluate_blockmodel(bm, truth, with_table=True)
        o = O.evaluate(a, truth)
        assert np.array_equal(ev["table"], o["table"])
        assert ev["accuracy"] == pytest.approx(o["accuracy"], abs=0)
        assert ev["f1_score"] == pytest.approx(o["f1"], rel=1e-12)
        assert ev["nmi"] == pytest.approx(o["nmi"], rel=1e-10)
        if unknown:
            assert np.isnan(ev["true_mdl"])
        else:
            labels = np.unique(truth, return_inverse=True)[1].astype(np.int32)   # MDL does not depend on labels
            tb = O.Blockmodel(O.Graph(V, s, d), ev["true_num_blocks"], labels)
            assert ev["true_mdl"] == pytest.approx(tb.mdl(), rel=1e-9)
