"""Seeded-replay parity against the reference itself.

A patched copy of the reference (oracle/_ref/replay/ref_driver, made by
oracle/build_reference.py from the reference's own sources: seeded engines, a log of every
proposal and accept uniform it draws, FP64 log terms, one orientation and a stable order for
merges of equal delta-MDL, an optional sweep cap) runs sbp::stochastic_block_partition and logs
the blockmodel at the start and end of every merge and finetune call.  The GPU engine replays
that stream through the C ABI:

  * call by call (sbp_finetune_replayed / sbp_merge_blocks_replayed), each call started from the
    reference's own start state: the end state (assignment, block matrix, d_out, d_in, d), the
    sweep count, every block's best merge and its delta-MDL must match;
  * as a whole partition (sbp_partition_replayed: the engine's own merge, finetune and
    golden-section steps, fed only the recorded proposals and uniforms): the block count after
    every call and the final assignment must match.

Integer state bit-exact; delta-MDL and MDL within 1e-9 relative (FP64 log terms on both sides).
The reference runs here on the host cores (its build travels with the repository's built files).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
RTOL_MDL = 1e-9


@pytest.fixture(scope="module")
def RR():
    import build_reference
    import ref_replay
    if not build_reference.replay_built():
        if not build_reference.reference_available():
            pytest.fail("oracle/_ref/replay/ref_driver is not built and the reference sources are absent: "
                        "run __graft_entry__.build() where the reference checkout is available")
        build_reference.build_replay()
    return ref_replay


def graph_of(cfg):
    import dcsbm
    return dcsbm.config_graph(cfg)


def assert_state(S, bm, state, what):
    assert bm.B == state["B"], what
    assert np.array_equal(bm.block_assignment(), state["assignment"]), what + ": assignment"
    import ref_replay
    assert np.array_equal(bm.blockmatrix(), ref_replay.matrix(state)), what + ": block matrix"
    do, di, d = bm.degrees_all()
    assert np.array_equal(do, state["d_out"]), what + ": d_out"
    assert np.array_equal(di, state["d_in"]), what + ": d_in"
    assert np.array_equal(d, state["d"]), what + ": d"


def engine_graph(S, V, src, dst, split):
    """The graph with the reference's own high/low degree split (its order of equal degrees)."""
    g = S.Graph(V, src, dst)
    g.set_split(*split)
    return g


def replay_calls_one_by_one(S, O, RR, V, src, dst, calls, split, batches=10, max_sweeps=0):
    """Every logged call replayed from the reference's start state; returns the calls checked."""
    g = engine_graph(S, V, src, dst, split)
    og = O.Graph(V, src, dst)
    checked = {"merge": 0, "finetune": 0}
    for c in calls:
        st0, st1 = c["begin"], c["end"]
        bm = S.Blockmodel(g, st0["B"], st0["assignment"])
        if c["kind"] == "merge":
            bm.setNum_blocks_to_merge(st0["num_blocks_to_merge"])
            out = S.block_merge.merge_blocks_replayed(bm, RR.merge_stream(c))
            best, delta = c["scores"]
            assert np.array_equal(out["best"], best), f"call {c['id']}: best merge per block"
            np.testing.assert_allclose(out["dS"], delta, rtol=RTOL_MDL, atol=RTOL_MDL * np.abs(delta).max())
            assert_state(S, bm, st1, f"merge call {c['id']} (B {st0['B']} -> {st1['B']})")
            checked["merge"] += 1
        else:
            # the start state of a finetune is a fresh rebuild (it follows a merge), d included
            assert_state(S, bm, st0, f"finetune call {c['id']} start")
            prop, uni = RR.finetune_stream(c, V)
            st = S.finetune.replayed(bm, c["kind"], prop, uni, batches=batches, bracket=c["bracket"] == 1,
                                     max_sweeps=max_sweeps)
            assert st["sweeps"] == c["sweeps"], f"finetune call {c['id']}: sweeps"
            assert_state(S, bm, st1, f"{c['kind']} call {c['id']} at B {st0['B']}")
            mdl = S.entropy.mdl(bm)
            ref = O.Blockmodel(og, st1["B"], st1["assignment"]).mdl()
            assert mdl == pytest.approx(ref, rel=RTOL_MDL)
            assert np.float32(mdl) == pytest.approx(st1["overall_entropy"], rel=1e-6)
            checked["finetune"] += 1
    return checked


def replay_whole_partition(S, RR, V, src, dst, calls, split, algo, batches=10, max_sweeps=0):
    g = engine_graph(S, V, src, dst, split)
    streams = [(RR.merge_stream(c), None) if c["kind"] == "merge" else RR.finetune_stream(c, V) for c in calls]
    out, st, counts = S.sbp.stochastic_block_partition_replayed(g, streams, algorithm=algo, batches=batches,
                                                                max_sweeps=max_sweeps)
    assert list(counts) == [c["end"]["B"] for c in calls], "block count after every call"
    return out, st


@pytest.mark.parametrize("algo", ["metropolis_hastings", "async_gibbs", "hybrid_mcmc"])
def test_replayed_calls_match_the_reference_call_by_call(S, O, RR, algo):
    V, src, dst, _ = graph_of(1)
    res, calls = RR.run("sbp", V, src, dst, algo=algo, seed=11)
    checked = replay_calls_one_by_one(S, O, RR, V, src, dst, calls, res["split"])
    assert checked["merge"] >= 5 and checked["finetune"] >= 5


@pytest.mark.parametrize("algo", ["metropolis_hastings", "async_gibbs", "hybrid_mcmc"])
def test_replayed_partition_matches_the_reference(S, O, RR, algo):
    V, src, dst, truth = graph_of(1)
    res, calls = RR.run("sbp", V, src, dst, algo=algo, seed=12)
    out, st = replay_whole_partition(S, RR, V, src, dst, calls, res["split"], algo)
    # the partition returns the triplet's best blockmodel, as the reference's loop does
    assert st["num_blocks"] == res["num_blocks"]
    assert st["mdl"] == pytest.approx(res["mdl"], rel=1e-6)
    assert np.array_equal(out, res["assignment"])


@pytest.mark.parametrize("algo,sweeps", [("async_gibbs", 3), ("hybrid_mcmc", 2), ("metropolis_hastings", 1)])
def test_replayed_partition_matches_the_reference_at_20k_vertices(S, O, RR, algo, sweeps):
    """The 20,000-vertex, 32-block benchmark graph, every finetune call capped at a few sweeps
    on both sides (the reference's MAX_NUM_ITERATIONS patched to the same cap)."""
    V, src, dst, _ = graph_of(2)
    res, calls = RR.run("sbp", V, src, dst, algo=algo, seed=13, max_sweeps=sweeps)
    out, st = replay_whole_partition(S, RR, V, src, dst, calls, res["split"], algo, max_sweeps=sweeps)
    assert st["num_blocks"] == res["num_blocks"]
    assert np.array_equal(out, res["assignment"])
