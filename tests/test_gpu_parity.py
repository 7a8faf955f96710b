"""GPU parity tests: the CUDA engine (through the C ABI) against the CPU oracle.

Integer state (assignment, block matrix, d_out, d_in, d, counters) must be bit-exact; delta-MDL
and MDL (FP64 log terms) within 1e-9 relative; the Hastings correction within 1e-12 relative.
Random numbers are identical on both sides (Philox4x32-10 or a replayed stream).
"""
import numpy as np
import pytest

from conftest import random_assignment, random_graph, random_records, toy_fixture

pytestmark = pytest.mark.gpu
RTOL_MDL = 1e-9


@pytest.fixture(params=["dense", "hashed"])
def storage(request, S):
    """Run the test with dense B x B counts and again with the row-hashed block matrix."""
    S.set_option("dense_max_blocks", 131072 if request.param == "dense" else 1)
    yield request.param
    S.set_option("dense_max_blocks", 131072)


def pair(S, O, V, s, d, B, a):
    g, og = S.Graph(V, s, d), O.Graph(V, s, d)
    return g, og, S.Blockmodel(g, B, a), O.Blockmodel(og, B, a)


def assert_same_state(bm, obm):
    assert bm.B == obm.B
    assert np.array_equal(bm.block_assignment(), obm.assignment())
    assert np.array_equal(bm.blockmatrix(), obm.matrix())
    do, di, d = bm.degrees_all()
    odo, odi, od = obm.degrees()
    assert np.array_equal(do, odo)
    assert np.array_equal(di, odi)
    assert np.array_equal(d, od)


def test_toy_known_answers_on_gpu(S, O):
    fx = toy_fixture()
    e = np.array(fx["edges"], np.int32)
    g = S.Graph(fx["num_vertices"], e[:, 0], e[:, 1])
    assert g.E == 23
    bm = S.Blockmodel(g, 3, np.array(fx["assignment"], np.int32))
    assert S.entropy.mdl(bm) == pytest.approx(fx["mdl"], rel=1e-6)
    do, di, d = bm.degrees_all()
    assert list(do) == [8, 7, 8] and list(di) == [9, 7, 7] and list(d) == [10, 9, 9]
    M0 = bm.blockmatrix()
    bm.move_vertex(7, 0)
    diff = bm.blockmatrix() - M0
    for k, v in fx["delta_move_7_to_0_with_self_in"].items():
        r, c = map(int, k.split(","))
        assert diff[r, c] == v


def test_complex_move_matches_oracle(S, O, storage):
    fx = toy_fixture()
    e = np.array(fx["edges"], np.int32)
    a = np.array(fx["complex_assignment"], np.int32)
    g, og, bm, obm = pair(S, O, 11, e[:, 0], e[:, 1], 6, a)
    bm.move_vertex(6, 0)
    obm.move_vertex(6, 0)
    assert_same_state(bm, obm)
    assert list(bm.degrees()) == [11, 7, 4, 7, 5, 6]


@pytest.mark.parametrize("V,K,B,seed", [(60, 3, 5, 1), (500, 6, 40, 2), (2000, 10, 300, 3), (3000, 20, 1200, 4)])
def test_mdl_matches_oracle(S, O, storage, V, K, B, seed):
    V, s, d, _ = random_graph(V, K, seed)
    a = random_assignment(V, B, seed)
    g, og, bm, obm = pair(S, O, V, s, d, B, a)
    assert_same_state(bm, obm)
    assert S.entropy.mdl(bm) == pytest.approx(obm.mdl(), rel=RTOL_MDL)


@pytest.mark.parametrize("V,K,B,seed", [(300, 5, 12, 1), (1500, 8, 200, 2), (800, 6, 3, 3)])
def test_evaluate_vertices_matches_oracle(S, O, storage, V, K, B, seed):
    V, s, d, _ = random_graph(V, K, seed)
    a = random_assignment(V, B, seed)
    g, og, bm, obm = pair(S, O, V, s, d, B, a)
    verts = np.arange(V, dtype=np.int32)
    rec = random_records(V, seed + 100)
    ps, dS, H, acc = bm.evaluate_vertices(verts, rec)
    n_moved = 0
    for v in range(V):
        ev = obm.eval_vertex(v, rec[v])
        assert ps[v] == ev["s"], v
        if ev["moved"]:
            n_moved += 1
            assert dS[v] == pytest.approx(ev["dS"], rel=RTOL_MDL, abs=1e-9), v
            assert H[v] == pytest.approx(ev["H"], rel=1e-12), v
            assert bool(acc[v]) == ev["accepted"], v
        else:
            assert not acc[v]
    assert n_moved > V // 4


@pytest.mark.parametrize("algo", ["metropolis_hastings", "asynchronous_gibbs", "hybrid_mcmc"])
@pytest.mark.parametrize("V,K,B,batches,seed", [(400, 5, 20, 4, 11), (1200, 8, 150, 10, 12), (900, 6, 6, 3, 13)])
def test_finetune_bit_exact(S, O, storage, algo, V, K, B, batches, seed):
    V, s, d, _ = random_graph(V, K, seed)
    a = random_assignment(V, B, seed)
    g, og, bm, obm = pair(S, O, V, s, d, B, a)
    code = {"metropolis_hastings": 0, "asynchronous_gibbs": 1, "hybrid_mcmc": 2}[algo]
    st = getattr(S.finetune, algo)(bm, batches=batches, seed=seed, call=3, max_sweeps=6)
    ost = obm.finetune(code, batches=batches, seed=seed, call=3, max_sweeps=6)
    assert_same_state(bm, obm)
    assert st["sweeps"] == ost["sweeps"]
    assert st["visits"] == ost["visits"]
    assert st["accepted"] == ost["accepted"]
    assert st["proposals_moved"] == ost["proposals_moved"]
    assert st["mdl"] == pytest.approx(ost["mdl"], rel=1e-7)   # both stored as float


@pytest.mark.parametrize("algo", [0, 1, 2])
def test_finetune_replay_bit_exact(S, O, storage, algo):
    V, s, d, _ = random_graph(700, 6, 21)
    a = random_assignment(V, 30, 21)
    g, og, bm, obm = pair(S, O, V, s, d, 30, a)
    sweeps = 5
    rec = random_records(sweeps * V, 77)
    st = S.finetune.run(bm, algo, batches=5, replay=rec, max_sweeps=sweeps)
    ost = obm.finetune(algo, batches=5, replay=rec, max_sweeps=sweeps)
    assert_same_state(bm, obm)
    assert st["accepted"] == ost["accepted"] and st["visits"] == ost["visits"]


def test_replay_too_short_is_an_error(S):
    V, s, d, _ = random_graph(200, 4, 5)
    g = S.Graph(V, s, d)
    bm = S.Blockmodel(g, 10, random_assignment(V, 10, 5))
    with pytest.raises(S.SbpError) as e:
        S.finetune.asynchronous_gibbs(bm, batches=2, replay=random_records(V // 2, 1), max_sweeps=2)
    assert e.value.code == 4


@pytest.mark.parametrize("approximate", [True, False])
@pytest.mark.parametrize("V,K,B,merge,seed", [(500, 5, 60, 30, 31), (1500, 8, 700, 350, 32), (300, 4, 9, 4, 33)])
def test_merge_blocks_bit_exact(S, O, storage, approximate, V, K, B, merge, seed):
    V, s, d, _ = random_graph(V, K, seed)
    a = random_assignment(V, B, seed)
    g, og, bm, obm = pair(S, O, V, s, d, B, a)
    bm.setNum_blocks_to_merge(merge)
    obm.set_num_blocks_to_merge(merge)
    res = S.block_merge.merge_blocks(bm, approximate=approximate, seed=seed, call=2)
    ores = obm.merge_blocks(approximate=approximate, seed=seed, call=2)
    assert np.array_equal(res["best"], ores["best"])
    np.testing.assert_allclose(res["dS"], ores["dS"], rtol=RTOL_MDL, atol=1e-9)
    assert res["merge_avoided"] == ores["avoided"]
    assert_same_state(bm, obm)


def test_merge_replay_bit_exact(S, O):
    V, s, d, _ = random_graph(600, 6, 41)
    a = random_assignment(V, 80, 41)
    g, og, bm, obm = pair(S, O, V, s, d, 80, a)
    rec = random_records(80 * 10, 5)
    bm.setNum_blocks_to_merge(40)
    obm.set_num_blocks_to_merge(40)
    res = S.block_merge.merge_blocks(bm, replay=rec)
    ores = obm.merge_blocks(replay=rec)
    assert np.array_equal(res["best"], ores["best"])
    assert_same_state(bm, obm)


@pytest.mark.parametrize("algo", ["metropolis_hastings", "async_gibbs", "hybrid_mcmc"])
def test_partition_bit_exact(S, O, storage, algo):
    V, s, d, truth = random_graph(500, 5, 51, kmin=6, kmax=40, w=0.85, alpha=10.0)
    g, og = S.Graph(V, s, d), O.Graph(V, s, d)
    out, st = S.sbp.stochastic_block_partition(g, algorithm=algo, batches=5, seed=9)
    code = {"metropolis_hastings": 0, "async_gibbs": 1, "hybrid_mcmc": 2}[algo]
    oout, ost = O.sbp(og, algo=code, batches=5, seed=9)
    assert np.array_equal(out, oout)
    assert st["num_blocks"] == ost["num_blocks"]
    assert st["mdl"] == ost["mdl"]
    assert st["visits"] == ost["visits"] and st["accepted"] == ost["accepted"]
    assert O.nmi(out, truth) > 0.8


def test_edge_cases(S, O, storage):
    # isolated vertices and a vertex with only a self loop
    s = np.array([0, 1, 2, 5, 5, 6], np.int32)
    d = np.array([1, 2, 0, 5, 6, 5], np.int32)
    V = 8
    a = np.array([0, 1, 2, 0, 1, 2, 0, 1], np.int32)
    g, og, bm, obm = pair(S, O, V, s, d, 3, a)
    assert g.E == 6
    for algo in (0, 1, 2):
        st = S.finetune.run(bm, algo, batches=2, seed=3, max_sweeps=3)
        ost = obm.finetune(algo, batches=2, seed=3, max_sweeps=3)
        assert_same_state(bm, obm)
        assert st["accepted"] == ost["accepted"]
    # B == 1: finetune is a no-op (src/finetune.cpp:33-35)
    one = S.Blockmodel(g, 1, np.zeros(V, np.int32))
    st = S.finetune.metropolis_hastings(one, seed=1)
    assert st["sweeps"] == 0 and np.all(one.block_assignment() == 0)
    # duplicate edges are dropped, first occurrence kept
    g2 = S.Graph(3, np.array([0, 0, 1, 0], np.int32), np.array([1, 1, 2, 1], np.int32))
    assert g2.E == 2


def test_invalid_arguments_raise(S):
    with pytest.raises(S.SbpError) as e:
        S.Graph(3, np.array([0, 5], np.int32), np.array([1, 2], np.int32))
    assert e.value.code == 1
    g = S.Graph(3, np.array([0, 1], np.int32), np.array([1, 2], np.int32))
    with pytest.raises(S.SbpError):
        S.Blockmodel(g, 2, np.array([0, 1, 2], np.int32))
    bm = S.Blockmodel(g, 2, np.array([0, 1, 1], np.int32))
    with pytest.raises(S.SbpError):
        bm.move_vertex(0, 7)


def test_config2_sweeps_keep_invariants(S, O):
    """20k-vertex, 32-block graph: after Gibbs and hybrid sweeps the counts equal a rebuild and
    the MDL equals the MDL of the rebuilt blockmodel (size-independent properties)."""
    import dcsbm
    V, s, d, truth = dcsbm.config_graph(2)
    g = S.Graph(V, s, d)
    a = random_assignment(V, 64, 2)
    bm = S.Blockmodel(g, 64, a)
    for algo in ("asynchronous_gibbs", "hybrid_mcmc", "metropolis_hastings"):
        getattr(S.finetune, algo)(bm, batches=10, seed=5, max_sweeps=2)
        rebuilt = S.Blockmodel(g, 64, bm.block_assignment())
        assert np.array_equal(bm.blockmatrix(), rebuilt.blockmatrix())
        do, di, _ = bm.degrees_all()
        rdo, rdi, _ = rebuilt.degrees_all()
        assert np.array_equal(do, rdo) and np.array_equal(di, rdi)
        assert S.entropy.mdl(bm) == pytest.approx(S.entropy.mdl(rebuilt), rel=1e-12)


def test_hashed_rows_grow_and_stay_exact(S, O):
    """Finetune from many tiny blocks on the row-hashed matrix: rows fill up as blocks grow,
    the storage is rebuilt with more room, and the chain stays bit-exact with the oracle."""
    S.set_option("dense_max_blocks", 1)
    S.set_option("hashed_row_factor", 2)   # tight rows: overflows are frequent
    try:
        V, s, d, _ = random_graph(2000, 8, 61, kmin=6, kmax=60, w=0.8)
        a = random_assignment(V, 900, 61)
        g, og, bm, obm = pair(S, O, V, s, d, 900, a)
        total = 0
        for algo in (1, 2, 0):
            st = S.finetune.run(bm, algo, batches=4, seed=algo + 3, call=algo, max_sweeps=8)
            ost = obm.finetune(algo, batches=4, seed=algo + 3, call=algo, max_sweeps=8)
            assert_same_state(bm, obm)
            assert st["accepted"] == ost["accepted"]
            total += st["overflow_rebuilds"]
        assert total > 0, "the test no longer drives the rows past their capacity"
    finally:
        S.set_option("dense_max_blocks", 131072)
        S.set_option("hashed_row_factor", 4)


def _reference_runs():
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "reference_runs.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("run", _reference_runs(), ids=lambda r: f"cfg{r['config']}-{r['algorithm']}")
def test_end_to_end_against_recorded_reference_runs(S, O, run):
    """Unseeded end-to-end criterion: the engine's final MDL within 0.5 % and its NMI against
    the planted blocks within 0.01 of a run of the reference itself (built from its sources;
    recorded by tests/golden/make_reference_runs.py)."""
    import dcsbm
    V, s, d, truth = dcsbm.config_graph(run["config"])
    g = S.Graph(V, s, d)
    assert g.E == run["E"]
    out, st = S.sbp.stochastic_block_partition(g, algorithm=run["algorithm"], batches=run["batches"],
                                               approximate=run["approximate"], seed=17)
    assert abs(st["mdl"] - run["mdl"]) <= 0.005 * run["mdl"]
    assert abs(O.nmi(out, truth) - run["nmi"]) <= 0.01


@pytest.mark.parametrize("batches,seed", [(10, 3), (3, 4), (7, 5)])   # odd batch counts flip the moved-slot parity
def test_graph_run_sweeps_equal_host_driven_sweeps(S, O, batches, seed):
    """An asynchronous-Gibbs finetune as one CUDA graph launch (loop and early stop on the GPU)
    gives the host-driven loop's chain, sweep count and counters, and the oracle's."""
    V, s, d, _ = random_graph(1500, 8, 90 + seed)
    a = random_assignment(V, 40, seed)
    g = S.Graph(V, s, d)
    res = []
    for mode in (1, 0):
        S.set_option("graph_sweeps", mode)
        try:
            bm = S.Blockmodel(g, 40, a)
            st = S.finetune.asynchronous_gibbs(bm, batches=batches, seed=seed, call=1)
            res.append((bm, st))
        finally:
            S.set_option("graph_sweeps", 1)
    (b1, s1), (b0, s0) = res
    assert np.array_equal(b1.block_assignment(), b0.block_assignment())
    assert np.array_equal(b1.blockmatrix(), b0.blockmatrix())
    assert np.array_equal(b1.degrees_all()[2], b0.degrees_all()[2])
    for k in ("sweeps", "visits", "accepted", "proposals_moved", "mdl"):
        assert s1[k] == s0[k], k
    obm = O.Blockmodel(O.Graph(V, s, d), 40, a)
    ost = obm.finetune(1, batches=batches, seed=seed, call=1)
    assert_same_state(b1, obm)
    assert s1["sweeps"] == ost["sweeps"]


@pytest.mark.parametrize("algo", [0, 1, 2])
@pytest.mark.parametrize("B,seed", [(7, 1), (64, 2), (128, 3), (129, 4), (700, 5), (2500, 6)])
def test_group_kernel_equals_warp_kernel(S, O, B, seed, algo):
    """The group kernels (groups of lanes per vertex; direct-indexed histograms up to 128 blocks,
    per-group hash tables and a chunked walk above; asynchronous-Gibbs batches and the
    Metropolis-Hastings rounds, hybrid using both) and the warp-per-vertex kernels give the same
    chain: same proposals, accept decisions and state, and both equal the oracle."""
    V, s, d, _ = random_graph(4000, 10, 90 + seed, kmin=4, kmax=60)
    a = random_assignment(V, B, seed)
    g = S.Graph(V, s, d)
    states = []
    for small in (2, 0):   # the group kernels at every B, then the warp kernels
        S.set_option("group_kernel", small)
        try:
            bm = S.Blockmodel(g, B, a)
            st = S.finetune.run(bm, algo, batches=5, seed=seed, call=3, max_sweeps=4)
            states.append((bm, st))
        finally:
            S.set_option("group_kernel", 1)
    (b1, s1), (b2, s2) = states
    assert np.array_equal(b1.block_assignment(), b2.block_assignment())
    assert np.array_equal(b1.blockmatrix(), b2.blockmatrix())
    assert s1["accepted"] == s2["accepted"] and s1["visits"] == s2["visits"]
    obm = O.Blockmodel(O.Graph(V, s, d), B, a)
    obm.finetune(algo, batches=5, seed=seed, call=3, max_sweeps=4)
    assert_same_state(b1, obm)


def test_device_ingest_keeps_the_first_occurrence_order(S, O):
    """Graph ingest on the device with many repeated (src, dst) pairs and self loops spread far
    apart in the input (so duplicates are resolved across CTAs): the degree split (degrees, ties by
    id) equals the oracle's, and the adjacency order, which the proposal's neighbour index reads,
    is the oracle's insert_nodup order: finetunes from the same start stay bit-exact."""
    V, s, d, _ = random_graph(3000, 8, 77, kmin=4, kmax=40)
    rng = np.random.default_rng(77)
    n = len(s)
    dup = rng.integers(0, n, 4 * n)            # every edge repeated about four times, shuffled in
    loops = rng.integers(0, V, 200).astype(np.int32)
    src = np.concatenate([s, s[dup], loops, loops[::-1]]).astype(np.int32)
    dst = np.concatenate([d, d[dup], loops, loops[::-1]]).astype(np.int32)
    g, og = S.Graph(V, src, dst), O.Graph(V, src, dst)
    assert g.E == og.E
    hi, lo = g.split()
    ohi, olo = og.split()
    assert np.array_equal(hi, ohi) and np.array_equal(lo, olo)
    a = random_assignment(V, 40, 77)
    for algo in (0, 1):
        bm, obm = S.Blockmodel(g, 40, a), O.Blockmodel(og, 40, a)
        st = S.finetune.run(bm, algo, batches=4, seed=9, call=algo, max_sweeps=3)
        ost = obm.finetune(algo, batches=4, seed=9, call=algo, max_sweeps=3)
        assert_same_state(bm, obm)
        assert st["accepted"] == ost["accepted"]
