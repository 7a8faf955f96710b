"""CPU checks of the patched reference build that records the replay stream
(oracle/build_reference.py, oracle/ref_replay/): every patch anchor applies, and the log of a
small partition is self-consistent -- calls alternate merge / finetune, each finetune call
holds one proposal record per vertex visit, and every logged end state's block matrix and
degrees equal a rebuild from its assignment (d excepted: it drifts by the reference's rule).
"""
import numpy as np
import pytest

from conftest import random_graph


@pytest.fixture(scope="module")
def RR():
    import build_reference as R
    if not R.replay_built():
        if not R.reference_available():
            pytest.fail("oracle/_ref/replay/ref_driver is not built and the reference sources are absent")
        R.build_replay()
    import ref_replay
    return ref_replay


def rebuild(V, src, dst, a, B):
    keep = {}
    for s, d in zip(src.tolist(), dst.tolist()):
        keep.setdefault((s, d), True)
    e = np.array(list(keep.keys()), np.int64)
    M = np.zeros((B, B), np.int64)
    np.add.at(M, (a[e[:, 0]], a[e[:, 1]]), 1)
    return M


@pytest.mark.parametrize("algo", ["metropolis_hastings", "async_gibbs", "hybrid_mcmc"])
def test_replay_log_is_consistent(RR, algo):
    V, s, d, _ = random_graph(400, 6, 21, kmin=4, kmax=30)
    res, calls = RR.run("sbp", V, s, d, algo=algo, threads=4, seed=3, batches=4)
    assert len(calls) >= 4
    assert [c["kind"] == "merge" for c in calls[::2]] == [True] * len(calls[::2])
    high, low = res["split"]
    assert len(high) + len(low) == V and len(set(high.tolist()) | set(low.tolist())) == V
    for c in calls:
        st0, st1 = c["begin"], c["end"]
        M = rebuild(V, s, d, st1["assignment"], st1["B"])
        assert np.array_equal(M, RR.matrix(st1))
        assert np.array_equal(M.sum(1), st1["d_out"]) and np.array_equal(M.sum(0), st1["d_in"])
        if c["kind"] == "merge":
            assert st1["B"] == st0["B"] - st0["num_blocks_to_merge"]
            assert c["scores"] is not None and len(c["scores"][0]) == st0["B"]
            assert len(c["merge"]) == 10 * st0["B"]
        else:
            assert st1["B"] == st0["B"] and 1 <= c["sweeps"] <= 100
            # every vertex is visited once per sweep (the async-Gibbs tail batch aside)
            assert len(c["visits"]) <= c["sweeps"] * V
            assert len(c["visits"]) >= c["sweeps"] * (V - V // 4 - 1)
            prop, uni = RR.finetune_stream(c, V)
            moved = prop[prop >= 0]
            assert moved.max() < st0["B"]
            assert np.all((uni[uni < 2.0] >= 0.0) & (uni[uni < 2.0] < 1.0))
