"""CPU pin of the oracle against the reference itself under seeded replay.

A patched copy of the reference (oracle/_ref/replay/ref_driver, built by oracle/build_reference.py
from the reference's own sources: seeded engines, a log of every proposal and accept uniform it
draws, FP64 log terms, one orientation and a stable order for merges of equal delta-MDL) runs
sbp::stochastic_block_partition on the host and logs the blockmodel at the start and end of every
merge and finetune call.  The C oracle replays each call from the reference's own start state,
fed only the reference's recorded proposals and accept uniforms:

  * merge calls: every block's best merge and its delta-MDL, then the state after the carry-out
    (simple, and the advanced priority-queue one) and rebuild;
  * finetune calls (all three algorithms, the reference's own order of equal degrees in the
    hybrid split): the sweep count and the end state, the drifting block degree d included;
  * whole partitions: the oracle's own merge, finetune and golden-section loop fed only the
    recorded streams, the block count after every call and the final assignment;
  * on the 20,000-vertex benchmark graph: finetunes of all three algorithms from a perturbed
    planted partition, and a 640 -> 320 block merge with both carry-outs.

Integer state bit for bit, delta-MDL within 1e-9 relative.  This checks the oracle's trajectory
rules (quirks Q1-Q5, the batch apply order, the early stops, the carry-out) against the reference
directly, without the GPU engine in between.
"""
import numpy as np
import pytest

RTOL_MDL = 1e-9


@pytest.fixture(scope="module")
def RR():
    import build_reference as R
    if not R.replay_built():
        if not R.reference_available():
            pytest.fail("oracle/_ref/replay/ref_driver is not built and the reference sources are absent")
        R.build_replay()
    import ref_replay
    return ref_replay


def assert_state(RR, bm, state, what):
    assert bm.B == state["B"], what
    assert np.array_equal(bm.assignment(), state["assignment"]), what + ": assignment"
    assert np.array_equal(bm.matrix(), RR.matrix(state)), what + ": block matrix"
    do, di, d = bm.degrees()
    assert np.array_equal(do, state["d_out"]), what + ": d_out"
    assert np.array_equal(di, state["d_in"]), what + ": d_in"
    assert np.array_equal(d, state["d"]), what + ": d"


@pytest.mark.parametrize("algo,approximate", [("metropolis_hastings", True), ("async_gibbs", True),
                                              ("hybrid_mcmc", True), ("async_gibbs", False)])
def test_oracle_replays_the_reference_call_by_call(O, RR, algo, approximate):
    """approximate False: the advanced carry-out (block_merge::carry_out_best_merges_advanced,
    a priority queue with lazily re-evaluated merges)."""
    import dcsbm
    V, src, dst, _ = dcsbm.config_graph(1)
    res, calls = RR.run("sbp", V, src, dst, algo=algo, seed=11, approximate=approximate)
    og = O.Graph(V, src, dst)
    og.set_split(*res["split"])
    code = {"metropolis_hastings": O.MH, "async_gibbs": O.GIBBS, "hybrid_mcmc": O.HYBRID}
    checked = {"merge": 0, "finetune": 0}
    for c in calls:
        st0, st1 = c["begin"], c["end"]
        bm = O.Blockmodel(og, st0["B"], st0["assignment"])
        if c["kind"] == "merge":
            bm.set_num_blocks_to_merge(st0["num_blocks_to_merge"])
            out = bm.merge_blocks_replayed(RR.merge_stream(c), approximate=approximate)
            best, delta = c["scores"]
            assert np.array_equal(out["best"], best), f"call {c['id']}: best merge per block"
            np.testing.assert_allclose(out["dS"], delta, rtol=RTOL_MDL, atol=RTOL_MDL * np.abs(delta).max())
            assert_state(RR, bm, st1, f"merge call {c['id']} (B {st0['B']} -> {st1['B']})")
            checked["merge"] += 1
        else:
            # a finetune starts from a fresh rebuild (it follows a merge), d included
            assert_state(RR, bm, st0, f"finetune call {c['id']} start")
            prop, uni = RR.finetune_stream(c, V)
            st = bm.finetune_replayed(code[c["kind"]], prop, uni, batches=10, bracket=c["bracket"] == 1)
            assert st["sweeps"] == c["sweeps"], f"finetune call {c['id']}: sweeps"
            assert_state(RR, bm, st1, f"{c['kind']} call {c['id']} at B {st0['B']}")
            assert np.float32(bm.mdl()) == pytest.approx(st1["overall_entropy"], rel=1e-6)
            checked["finetune"] += 1
    assert checked["merge"] >= 5 and checked["finetune"] >= 5, checked


@pytest.mark.parametrize("algo,approximate,batches", [
    ("metropolis_hastings", True, 10), ("async_gibbs", True, 10), ("hybrid_mcmc", True, 10),
    ("metropolis_hastings", False, 10), ("async_gibbs", True, 3), ("hybrid_mcmc", True, 7)])
def test_oracle_replays_the_reference_partition(O, RR, algo, approximate, batches):
    """The oracle's own merge, finetune and golden-section loop, fed only the reference's
    recorded proposals and uniforms: the block count after every call, the final blockmodel's
    assignment and its MDL equal the reference's (batches 3 and 7 leave a tail that the
    reference's batch loop skips)."""
    import dcsbm
    V, src, dst, _ = dcsbm.config_graph(1)
    res, calls = RR.run("sbp", V, src, dst, algo=algo, seed=12, approximate=approximate, batches=batches)
    og = O.Graph(V, src, dst)
    og.set_split(*res["split"])
    streams = [(RR.merge_stream(c), None) if c["kind"] == "merge" else RR.finetune_stream(c, V) for c in calls]
    code = {"metropolis_hastings": O.MH, "async_gibbs": O.GIBBS, "hybrid_mcmc": O.HYBRID}
    out, st, counts = O.sbp_replayed(og, streams, algo=code[algo], batches=batches, approximate=approximate)
    assert list(counts) == [c["end"]["B"] for c in calls], "block count after every call"
    assert st["num_blocks"] == res["num_blocks"]
    assert st["mdl"] == pytest.approx(res["mdl"], rel=1e-6)
    assert np.array_equal(out, res["assignment"])


def _reference_runs(config):
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "reference_runs.json")) as f:
        return [r for r in json.load(f) if r["config"] == config]


@pytest.mark.parametrize("run", _reference_runs(1), ids=lambda r: r["algorithm"])
def test_oracle_meets_the_unseeded_criterion_against_the_unmodified_reference(O, run):
    """The oracle's own Philox-seeded partition of the 1,000-vertex graph against a run of the
    unmodified reference (FP32 logs, unseeded engines; tests/golden/reference_runs.json): final
    MDL within 0.5 % and NMI against the planted blocks within 0.01.  The documented departures
    (Philox draws, walk order, FP64 logs, the zero snap, rounded merge ranking) do not move the
    outcome out of the criterion."""
    import dcsbm
    V, s, d, truth = dcsbm.config_graph(1)
    og = O.Graph(V, s, d)
    assert og.E == run["E"]
    code = {"metropolis_hastings": O.MH, "async_gibbs": O.GIBBS, "hybrid_mcmc": O.HYBRID}
    out, st = O.sbp(og, algo=code[run["algorithm"]], batches=run["batches"], approximate=run["approximate"], seed=17)
    assert abs(st["mdl"] - run["mdl"]) <= 0.005 * run["mdl"]
    assert abs(O.nmi(out, truth) - run["nmi"]) <= 0.01


def _perturbed_planted(truth, frac, seed):
    rng = np.random.default_rng(seed)
    a = truth.astype(np.int32).copy()
    moved = rng.random(len(a)) < frac
    a[moved] = rng.integers(0, int(a.max()) + 1, moved.sum())
    return a


@pytest.mark.parametrize("algo", ["metropolis_hastings", "async_gibbs", "hybrid_mcmc"])
def test_oracle_replays_reference_finetunes_on_the_20k_graph(O, RR, algo):
    """The 20,000-vertex, 32-block benchmark graph from its planted partition with 30 % of the
    vertices moved: one reference finetune capped at 5 sweeps, replayed by the oracle bit for
    bit (thousands of accepted moves per call)."""
    import dcsbm
    V, src, dst, truth = dcsbm.config_graph(2)
    a = _perturbed_planted(truth, 0.3, 5)
    res, calls = RR.run("finetune", V, src, dst, algo=algo, assignment=a, seed=7, max_sweeps=5)
    og = O.Graph(V, src, dst)
    og.set_split(*res["split"])
    (c,) = [c for c in calls if c["kind"] != "merge"]
    code = {"metropolis_hastings": O.MH, "async_gibbs": O.GIBBS, "hybrid_mcmc": O.HYBRID}
    bm = O.Blockmodel(og, c["begin"]["B"], c["begin"]["assignment"])
    prop, uni = RR.finetune_stream(c, V)
    st = bm.finetune_replayed(code[algo], prop, uni, batches=10, bracket=c["bracket"] == 1, max_sweeps=5)
    assert st["sweeps"] == c["sweeps"]
    assert st["accepted"] > 1000
    assert_state(RR, bm, c["end"], f"{algo} on the 20k graph")


@pytest.mark.parametrize("approximate", [True, False])
def test_oracle_replays_a_reference_merge_on_the_20k_graph(O, RR, approximate):
    """A merge of the 20,000-vertex graph from 640 blocks (each planted block split 20 ways) to
    320, both carry-outs: every block's best merge and delta-MDL and the state after it."""
    import dcsbm
    V, src, dst, truth = dcsbm.config_graph(2)
    rng = np.random.default_rng(6)
    _, a = np.unique(truth.astype(np.int64) * 20 + rng.integers(0, 20, V), return_inverse=True)
    a = a.astype(np.int32)
    B = int(a.max()) + 1
    res, calls = RR.run("merge", V, src, dst, assignment=a, num_blocks_to_merge=B // 2, seed=8,
                        approximate=approximate)
    (c,) = [c for c in calls if c["kind"] == "merge"]
    bm = O.Blockmodel(O.Graph(V, src, dst), c["begin"]["B"], c["begin"]["assignment"])
    bm.set_num_blocks_to_merge(c["begin"]["num_blocks_to_merge"])
    out = bm.merge_blocks_replayed(RR.merge_stream(c), approximate=approximate)
    best, delta = c["scores"]
    assert np.array_equal(out["best"], best)
    np.testing.assert_allclose(out["dS"], delta, rtol=RTOL_MDL, atol=RTOL_MDL * np.abs(delta).max())
    assert_state(RR, bm, c["end"], "merge on the 20k graph")
