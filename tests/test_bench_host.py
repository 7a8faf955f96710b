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
