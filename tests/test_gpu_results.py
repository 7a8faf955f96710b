"""Intermediate records (sbp::add_intermediate, src/sbp.cpp:36-59) and the results CSV
(write_results, src/main.cpp:23-51) of a GPU partition, each figure checked against a numpy
restatement of the reference's own formula on the partition's assignment:
  Graph::modularity (src/graph.cpp:142-163, the O(V^2) pair sum, evaluated literally),
  Blockmodel::interblock_edges (src/blockmodel/blockmodel.cpp:257-261),
  Blockmodel::block_size_variation (src/blockmodel/blockmodel.cpp:9-27),
  entropy::mdl and normalize_mdl_v1 / v2 (src/entropy.cpp:559-589, the C oracle's mdl).
"""
import csv
import os

import numpy as np
import pytest

from conftest import random_graph

pytestmark = pytest.mark.gpu


def graph_lists(V, src, dst):
    seen, out_n, in_n = set(), [[] for _ in range(V)], [[] for _ in range(V)]
    for s, d in zip(src.tolist(), dst.tolist()):
        if (s, d) in seen:
            continue
        seen.add((s, d))
        out_n[s].append(d)
        in_n[d].append(s)
    return out_n, in_n, len(seen)


def modularity_pairs(V, out_n, in_n, E, a):
    A = np.zeros((V, V))
    for i in range(V):
        A[i, out_n[i]] = 1.0
    dout = np.array([len(x) for x in out_n], np.float64)
    din = np.array([len(x) for x in in_n], np.float64)
    same = a[:, None] == a[None, :]
    return float(((A - np.outer(dout, din) / E) * same).sum() / E)


def size_variation(a, B):
    sizes = np.bincount(a, minlength=B).astype(np.float64)
    mean = sizes.sum() / B
    var = ((sizes - mean) ** 2).sum() / B
    return float(np.float32(var / ((sizes.max() - sizes.min()) * (sizes.max() - mean) / 4.0)))


def test_partition_intermediates_and_csv(S, O, tmp_path):
    V, src, dst, truth = random_graph(600, 6, 41, kmin=5, kmax=40)
    g = S.Graph(V, src, dst)
    S.sbp.clear_intermediates()
    out, st = S.sbp.stochastic_block_partition(g, batches=4, seed=3)
    rec = S.sbp.get_intermediates()
    assert rec[0]["iteration"] == 0.0 and rec[0]["num_blocks"] == V
    assert rec[1]["iteration"] == 0.5 and rec[1]["num_blocks"] == V // 2
    assert [r["iteration"] for r in rec[2:-1]] == [float(k) for k in range(1, st["outer_iterations"] + 1)]
    final = rec[-1]
    assert final["iteration"] == -1.0 and final["num_blocks"] == st["num_blocks"]
    assert all(r["modularity"] == -1.0 for r in rec[:-1])
    out_n, in_n, E = graph_lists(V, src, dst)
    og = O.Graph(V, src, dst)
    assert final["modularity"] == pytest.approx(modularity_pairs(V, out_n, in_n, E, out), rel=1e-9, abs=1e-12)
    within = sum(1 for i in range(V) for j in out_n[i] if out[i] == out[j])
    assert final["interblock_edges"] == pytest.approx((E - within) / E, rel=1e-12)
    assert final["block_size_variation"] == pytest.approx(size_variation(out, st["num_blocks"]), rel=1e-6)
    assert final["mdl"] == pytest.approx(O.Blockmodel(og, st["num_blocks"], out).mdl(), rel=1e-6)
    assert rec[0]["normalized_mdl_v1"] == pytest.approx(rec[0]["mdl"] / O.null_mdl_v1(E), rel=1e-12)
    assert rec[0]["mdl"] == pytest.approx(O.Blockmodel(og, V, np.arange(V, dtype=np.int32)).mdl(), rel=1e-9)
    assert final["visits"] == st["visits"] and final["mcmc_iterations"] >= st["sweeps"]
    # the CSV in the reference's schema
    import sbp_results as R
    ev = S.evaluate.evaluate_blockmodel(S.Blockmodel(g, st["num_blocks"], out), truth)
    path = R.write_results(R.results_path(str(tmp_path) + "/", V, "dcsbm"), rec, num_vertices=V, num_edges=E,
                           algorithm="async_gibbs", evaluation=ev, runtime=st["total_seconds"], tag="test")
    rows = list(csv.reader(open(path), skipinitialspace=True))
    assert rows[0] == R.COLUMNS and len(rows) == len(rec) + 1
    assert float(rows[-1][R.COLUMNS.index("f1_score")]) == pytest.approx(ev["f1_score"])
    assert float(rows[-1][R.COLUMNS.index("iteration")]) == -1.0
