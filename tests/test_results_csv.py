"""CPU tests of the results CSV writer (sbp_results.py, the reference's write_results of
src/main.cpp:23-51): its null-model MDLs against the reference's known answers and the oracle,
the file layout, and one row per intermediate record with the header written once."""
import csv
import math

import pytest

from conftest import toy_fixture


def test_null_models_match_the_reference_known_answers(O):
    import sbp_results as R
    fx = toy_fixture()   # EntropyTest.NullModelMDL_v1 / _v2 (FP32 in the reference)
    assert R.null_mdl_v1(50) == pytest.approx(fx["null_mdl_v1_E50"], rel=1e-6)
    assert R.null_mdl_v2(10, 50) == pytest.approx(fx["null_mdl_v2_V10_E50"], rel=1e-6)
    for E, V in ((50, 10), (17_600, 1_000), (4_061_906, 200_000)):
        assert R.null_mdl_v1(E) == pytest.approx(O.null_mdl_v1(E), rel=1e-12)
        assert R.null_mdl_v2(V, E) == pytest.approx(O.null_mdl_v2(V, E), rel=1e-12)


def test_rows_follow_the_reference_schema(tmp_path):
    import sbp_results as R
    path = R.results_path(str(tmp_path / "csv") + "/", 600, "dcsbm")
    assert path.endswith("600/dcsbm.csv")
    recs = [dict(iteration=it, mdl=1000.0 - 10 * k, normalized_mdl_v1=0.5, normalized_mdl_v2=0.4, modularity=-1.0,
                 interblock_edges=0.3, block_size_variation=0.2, mcmc_iterations=7 * k, num_blocks=600 >> k,
                 visits=6000 * (k + 1), seconds=0.01 * (k + 1))
            for k, it in enumerate((0.0, 0.5, 1.0, -1.0))]
    ev = dict(f1_score=0.9, nmi=0.95, true_mdl=950.0)
    for _ in range(2):   # a second run appends its rows under the same header
        R.write_results(path, recs, num_vertices=600, num_edges=9000, algorithm="async_gibbs", evaluation=ev,
                        runtime=1.5, eval_kernel_gbps=40.0, hbm_peak_gbps=6524.3)
    with open(path) as f:
        rows = list(csv.reader(f, skipinitialspace=True))
    assert rows[0] == R.COLUMNS
    assert len(rows) == 1 + 2 * len(recs) and all(len(r) == len(R.COLUMNS) for r in rows[1:])
    col = {name: i for i, name in enumerate(R.COLUMNS)}
    for r, rec in zip(rows[1:], recs + recs):
        assert float(r[col["iteration"]]) == rec["iteration"]
        assert int(r[col["num_blocks"]]) == rec["num_blocks"]
        assert float(r[col["true_mdl_v1"]]) == pytest.approx(950.0 / R.null_mdl_v1(9000))
        assert float(r[col["true_mdl_v2"]]) == pytest.approx(950.0 / R.null_mdl_v2(600, 9000))
        assert float(r[col["vertex_moves_per_s"]]) == pytest.approx(rec["visits"] / rec["seconds"])
        assert float(r[col["eval_roofline_frac"]]) == pytest.approx(40.0 / 6524.3)
        assert r[col["algorithm"]] == "async_gibbs" and r[col["undirected"]] == "0"
    assert not math.isnan(float(rows[1][col["mdl"]]))
