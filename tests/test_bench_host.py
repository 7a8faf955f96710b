"""CPU tests of bench.py's host-side pieces: the reference sample's level order and the DRAM
traffic figure read from the committed profile summaries."""
import os
import sys

from conftest import ORACLE, ROOT


def test_halving_levels_and_spread_order():
    sys.path.insert(0, ORACLE)
    import build_reference as R
    levels = R.halving_levels(200_000, 71)
    assert levels[0] == 100_000 and levels[-1] == 71
    assert all(a > b for a, b in zip(levels, levels[1:]))
    for n in (1, 2, 5, 12, 16):
        order = R.spread_order(n)
        assert sorted(order) == list(range(n))
        assert order[0] == 0
    order = R.spread_order(len(levels))
    # the first few picks reach both halves of the schedule
    first = order[:3]
    assert min(first) < len(levels) // 2 <= max(first)


def test_profiled_traffic_comes_from_a_committed_summary():
    sys.path.insert(0, ROOT)
    import bench
    traffic, src = bench.profiled_traffic("k_gibbs_eval", 4)
    assert traffic is not None and traffic > 1e6
    assert src.startswith("profiles" + os.sep) and os.path.exists(os.path.join(ROOT, src))
    text = open(os.path.join(ROOT, src)).read()
    assert "ncu" in text and "--clock-control none" in text


def test_eval_load_model_counts_the_loads_of_a_visit():
    """On a tiny graph the model's neighbour and block counts equal a direct count, and its byte
    figures follow from them."""
    import numpy as np
    sys.path.insert(0, ROOT)
    import bench
    V = 6
    src = np.array([0, 0, 0, 1, 2, 3, 3, 0, 5], np.int32)   # a duplicate (0, 1) and a self loop (3, 3)
    dst = np.array([1, 2, 1, 2, 0, 3, 4, 3, 0], np.int32)
    truth = np.array([0, 0, 1, 1, 2, 2], np.int32)
    m = bench.eval_load_model(V, src, dst, truth, 1)          # one part per block: the planted blocks
    # neighbours after de-duplication (out lists keep the self loop, in lists drop it):
    # 0: out 1 2 3, in 2 5; 1: out 2, in 0; 2: out 0, in 0 1; 3: out 3 4, in 0; 4: in 3; 5: out 0
    k = [5, 2, 3, 3, 1, 1]
    assert m["mean_k"] == np.mean(k)
    # distinct blocks of the neighbours other than v itself
    nb = [3, 2, 1, 2, 1, 1]
    assert m["mean_distinct_neighbour_blocks"] == np.mean(nb)
    assert m["bytes_per_visit"]["formula"] == 12 + 8 * np.mean(k)
    assert m["B"] == 3 and m["ld"] == 128 and m["chunks_per_row"] == 1
    walk = 8 + 2 * 4 + 512
    assert m["bytes_per_visit"]["with_blockmodel"] == 16 + 1 + 4 + 8 * np.mean(k) + 20 * np.mean(nb) + 32 + walk
