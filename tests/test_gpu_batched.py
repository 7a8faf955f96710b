"""GPU tests of the batched partitioner: every graph of a batch gets exactly the partition that
sbp_partition gives it alone (assignment, block count, MDL and counters), whatever shapes the
autotuner picks, including rounds that fall back to the single-graph finetune."""
import numpy as np
import pytest

from conftest import random_graph

pytestmark = pytest.mark.gpu


def uneven_graphs(seed, sizes):
    out = []
    for i, V in enumerate(sizes):
        K = int(round(1.2 * V ** 0.35))
        out.append(random_graph(V, K, seed + i, kmin=6, kmax=60, w=0.55 + 0.05 * (i % 7), alpha=3.0))
    return out


def with_hub(V, s, d, hub=0, extra=400, seed=0):
    """Add in-edges to one vertex so that it is evaluated on the heavy path."""
    rng = np.random.default_rng(seed)
    src = rng.choice(np.arange(1, V), size=min(extra, V - 1), replace=False).astype(np.int32)
    return V, np.concatenate([s, src]), np.concatenate([d, np.full(len(src), hub, np.int32)])


def single(S, g, seed):
    return S.sbp.stochastic_block_partition(g, algorithm="async_gibbs", batches=10, seed=seed)


def assert_same(out_b, st_b, out_s, st_s):
    assert np.array_equal(out_b, out_s)
    for k in ("num_blocks", "mdl", "sweeps", "visits", "accepted", "proposals_moved", "outer_iterations"):
        assert st_b[k] == st_s[k], k


def test_batched_partitions_equal_the_oracle(S, O):
    """Each graph of a batch against the CPU oracle's own partition of it (same Philox stream):
    assignment, block count, sweeps, visits and accepted moves bit-exact, MDL within 1e-6 (the
    float overall entropy)."""
    specs = uneven_graphs(400, [350, 900, 1300, 600])
    graphs = [S.Graph(V, s, d) for V, s, d, _ in specs]
    outs, stats, info = S.batched.stochastic_block_partition(graphs, batches=10, seed=8)
    assert info["batched_finetunes"] > 0
    for (V, s, d, _), out, st in zip(specs, outs, stats):
        o_out, o_st = O.sbp(O.Graph(V, s, d), batches=10, seed=8)
        assert np.array_equal(out, o_out)
        assert st["num_blocks"] == o_st["num_blocks"] and st["sweeps"] == o_st["mcmc_sweeps"]
        assert st["visits"] == o_st["visits"] and st["accepted"] == o_st["accepted"]
        assert st["mdl"] == pytest.approx(o_st["mdl"], rel=1e-6)


def test_batched_equals_single_partitions(S):
    specs = uneven_graphs(100, [300, 1700, 800, 2500, 450, 1200])
    graphs = []
    for i, (V, s, d, _) in enumerate(specs):
        if i == 3:
            V, s, d = with_hub(V, s, d, seed=i)
        graphs.append(S.Graph(V, s, d))
    S.batched.reset_tuning()
    outs, stats, info = S.batched.stochastic_block_partition(graphs, batches=10, seed=5)
    assert info["tuned"] == 1 and info["candidates"] >= 1
    assert info["batched_finetunes"] > 0 and info["sweep_launches"] > 0
    for g, out, st in zip(graphs, outs, stats):
        out_s, st_s = single(S, g, 5)
        assert_same(out, st, out_s, st_s)
    # the tuned shape is reused, and the answer does not change
    outs2, stats2, info2 = S.batched.stochastic_block_partition(graphs, batches=10, seed=5)
    assert info2["tuned"] == 0
    for a, b in zip(outs, outs2):
        assert np.array_equal(a, b)


def test_batched_fallback_rounds_are_identical(S):
    """Small dense limit: the first rounds use row-hashed storage and the single-graph finetune."""
    specs = uneven_graphs(200, [900, 400, 1500])
    graphs = [S.Graph(V, s, d) for V, s, d, _ in specs]
    S.set_option("dense_max_blocks", 64)
    try:
        outs, stats, info = S.batched.stochastic_block_partition(graphs, batches=8, seed=11)
        assert info["fallback_finetunes"] > 0 and info["batched_finetunes"] > 0
        for g, out, st in zip(graphs, outs, stats):
            out_s, st_s = S.sbp.stochastic_block_partition(g, algorithm="async_gibbs", batches=8, seed=11)
            assert_same(out, st, out_s, st_s)
    finally:
        S.set_option("dense_max_blocks", 131072)


def test_batched_other_algorithms_fall_back(S):
    specs = uneven_graphs(300, [400, 700])
    graphs = [S.Graph(V, s, d) for V, s, d, _ in specs]
    outs, stats, info = S.batched.stochastic_block_partition(graphs, algorithm="hybrid_mcmc", batches=5, seed=3)
    assert info["batched_finetunes"] == 0 and info["fallback_finetunes"] > 0
    for g, out, st in zip(graphs, outs, stats):
        out_s, st_s = S.sbp.stochastic_block_partition(g, algorithm="hybrid_mcmc", batches=5, seed=3)
        assert_same(out, st, out_s, st_s)


def test_batched_single_graph_and_errors(S):
    V, s, d, _ = random_graph(600, 5, 9)
    g = S.Graph(V, s, d)
    outs, stats, _ = S.batched.stochastic_block_partition([g], seed=2)
    out_s, st_s = single(S, g, 2)
    assert_same(outs[0], stats[0], out_s, st_s)
    with pytest.raises(S.SbpError):
        S.batched.stochastic_block_partition([g], batches=0)


def test_batched_wait_runs_out_and_the_library_stays_usable(S):
    """Failure detection without a GPU fault: a graph's sweep queue is made on the host so that it
    never opens (sbp_set_option "batched_stall_graph"); the persistent CTAs' bounded idle wait
    (set short here) runs out, the call fails with SBP_ERR_DEVICE naming the wait, and the next
    call on the same context succeeds."""
    graphs = [S.Graph(*random_graph(600, 5, 301)[:3]), S.Graph(*random_graph(800, 6, 302)[:3])]
    S.set_option("batched_wait_limit", 4096)
    S.set_option("batched_stall_graph", 1)
    try:
        with pytest.raises(S.SbpError) as e:
            S.batched.stochastic_block_partition(graphs, batches=4, seed=3)
        assert e.value.code == 5 and "wait limit" in str(e.value)
    finally:
        S.set_option("batched_stall_graph", -1)
        S.set_option("batched_wait_limit", 1 << 22)
    outs, _, _ = S.batched.stochastic_block_partition(graphs, batches=4, seed=3)
    for g, out in zip(graphs, outs):
        single, _ = S.sbp.stochastic_block_partition(g, batches=4, seed=3)
        assert np.array_equal(out, single)


@pytest.mark.parametrize("overlap,threads", [(0, 1), (16, 1), (1024, 1), (0, 8), (64, 8), (64, 3)])
def test_batched_overlapped_merges_are_identical(S, overlap, threads):
    """The graphs between finetunes are processed while a sweep launch runs (sbp_set_option
    "batched_overlap" = CTA slots left free for them; 1024 leaves half the grid, 0 runs them
    before the next launch instead), on a pool of host threads with a context each
    ("batched_threads"; 1: the calling thread on a second context): the partitions are the
    single-graph ones either way, including rounds on row-hashed storage with the single-graph
    finetune."""
    specs = uneven_graphs(500, [700, 2100, 350, 1500, 900, 3000, 1200, 500])
    graphs = [S.Graph(V, s, d) for V, s, d, _ in specs]
    S.set_option("batched_overlap", overlap)
    S.set_option("batched_threads", threads)
    S.set_option("dense_max_blocks", 256)
    try:
        outs, stats, info = S.batched.stochastic_block_partition(graphs, batches=10, seed=21)
        assert info["batched_finetunes"] > 0 and info["fallback_finetunes"] > 0
        assert info["serial_seconds"] > 0 and (overlap == 0) == (info["overlapped_seconds"] == 0)
        for g, out, st in zip(graphs, outs, stats):
            assert_same(out, st, *single(S, g, 21))
    finally:
        S.set_option("dense_max_blocks", 131072)
        S.set_option("batched_overlap", 64)
        S.set_option("batched_threads", 8)
