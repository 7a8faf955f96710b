"""GPU parity with the CPU oracle on the benchmark graphs themselves (not toy sizes):

  * the 20,000-vertex / 32-block graph: a few sweeps of Metropolis-Hastings, asynchronous Gibbs
    and hybrid on both storages (dense and row-hashed), from a perturbed planted partition and
    from a split one (B = 320);
  * one merge call on that graph at B = V / 2 (the partition's second merge round);
  * the 200,000-vertex / 71-block graph: two asynchronous-Gibbs sweeps from a perturbed planted
    partition;
  * row-hashed storage with tight rows at 20,000 vertices, where the rows overflow again and again.

Bit-exact integer state (assignment, block matrix, d_out, d_in, d) and counters; MDL within 1e-9.
"""
import numpy as np
import pytest

from conftest import random_assignment

pytestmark = pytest.mark.gpu
RTOL_MDL = 1e-9


@pytest.fixture(scope="module")
def cfg2():
    import dcsbm
    return dcsbm.config_graph(2)


@pytest.fixture(params=["dense", "hashed"])
def storage(request, S):
    S.set_option("dense_max_blocks", 131072 if request.param == "dense" else 1)
    yield request.param
    S.set_option("dense_max_blocks", 131072)


def perturbed(truth, frac, seed, K=None):
    rng = np.random.default_rng(seed)
    K = K or int(truth.max()) + 1
    a = truth.astype(np.int32).copy()
    f = rng.random(len(a)) < frac
    a[f] = rng.integers(0, K, f.sum())
    return a


def split(truth, parts, seed):
    rng = np.random.default_rng(seed)
    a = truth.astype(np.int64) * parts + rng.integers(0, parts, len(truth))
    return np.unique(a, return_inverse=True)[1].astype(np.int32)


def same_state(bm, obm):
    assert bm.B == obm.B
    assert np.array_equal(bm.block_assignment(), obm.assignment())
    assert np.array_equal(bm.blockmatrix(), obm.matrix())
    do, di, d = bm.degrees_all()
    odo, odi, od = obm.degrees()
    assert np.array_equal(do, odo) and np.array_equal(di, odi) and np.array_equal(d, od)


@pytest.mark.parametrize("algo,sweeps", [(0, 2), (1, 3), (2, 2)])
@pytest.mark.parametrize("start", ["perturbed", "split"])
def test_finetune_on_the_20k_graph(S, O, cfg2, storage, algo, sweeps, start):
    V, s, d, truth = cfg2
    a = perturbed(truth, 0.3, 7) if start == "perturbed" else split(truth, 10, 7)
    B = int(a.max()) + 1
    g, og = S.Graph(V, s, d), O.Graph(V, s, d)
    bm, obm = S.Blockmodel(g, B, a), O.Blockmodel(og, B, a)
    st = S.finetune.run(bm, algo, batches=10, seed=21, call=algo, max_sweeps=sweeps)
    ost = obm.finetune(algo, batches=10, seed=21, call=algo, max_sweeps=sweeps)
    same_state(bm, obm)
    assert st["sweeps"] == ost["sweeps"] and st["accepted"] == ost["accepted"] and st["visits"] == ost["visits"]
    assert S.entropy.mdl(bm) == pytest.approx(obm.mdl(), rel=RTOL_MDL)


def test_merge_round_at_half_the_vertices_on_the_20k_graph(S, O, cfg2):
    """A merge call at B = V / 2 (the partition's second round), from vertices paired at random."""
    V, s, d, truth = cfg2
    g, og = S.Graph(V, s, d), O.Graph(V, s, d)
    a = (np.random.default_rng(3).permutation(V) // 2).astype(np.int32)
    B = V // 2
    bm, obm = S.Blockmodel(g, B, a), O.Blockmodel(og, B, a)
    bm.setNum_blocks_to_merge(B // 2)
    obm.set_num_blocks_to_merge(B // 2)
    m = S.block_merge.merge_blocks(bm, seed=4, call=1)
    om = obm.merge_blocks(seed=4, call=1)
    assert np.array_equal(m["best"], om["best"])
    np.testing.assert_allclose(m["dS"], om["dS"], rtol=RTOL_MDL, atol=RTOL_MDL * np.abs(om["dS"]).max())
    assert bm.B == B - B // 2
    assert np.array_equal(bm.block_assignment(), obm.assignment())
    do, di, dd = bm.degrees_all()
    odo, odi, od = obm.degrees()
    assert np.array_equal(do, odo) and np.array_equal(di, odi) and np.array_equal(dd, od)


def test_two_gibbs_sweeps_on_the_200k_graph(S, O):
    import dcsbm
    V, s, d, truth = dcsbm.config_graph(4)
    a = perturbed(truth, 0.25, 9)
    B = int(truth.max()) + 1
    g, og = S.Graph(V, s, d), O.Graph(V, s, d)
    bm, obm = S.Blockmodel(g, B, a), O.Blockmodel(og, B, a)
    st = S.finetune.asynchronous_gibbs(bm, batches=10, seed=33, call=0, max_sweeps=2)
    ost = obm.finetune(1, batches=10, seed=33, call=0, max_sweeps=2)
    same_state(bm, obm)
    assert st["accepted"] == ost["accepted"] and st["accepted"] > 1000
    assert S.entropy.mdl(bm) == pytest.approx(obm.mdl(), rel=RTOL_MDL)


def test_hashed_rows_overflow_again_and_again_at_20k(S, O, cfg2):
    V, s, d, truth = cfg2
    S.set_option("dense_max_blocks", 1)
    S.set_option("hashed_row_factor", 2)
    try:
        B = 3000
        a = random_assignment(V, B, 5)
        g, og = S.Graph(V, s, d), O.Graph(V, s, d)
        bm, obm = S.Blockmodel(g, B, a), O.Blockmodel(og, B, a)
        total = 0
        for algo in (1, 2):
            st = S.finetune.run(bm, algo, batches=10, seed=algo + 40, call=algo, max_sweeps=4)
            ost = obm.finetune(algo, batches=10, seed=algo + 40, call=algo, max_sweeps=4)
            same_state(bm, obm)
            assert st["accepted"] == ost["accepted"]
            total += st["overflow_rebuilds"]
        assert total >= 3, "the rows no longer overflow repeatedly"
    finally:
        S.set_option("dense_max_blocks", 131072)
        S.set_option("hashed_row_factor", 4)
