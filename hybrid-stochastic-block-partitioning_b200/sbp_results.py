"""Results CSV of a partition run in the reference's schema (write_results, src/main.cpp:23-51),
with throughput columns added at the end.

One row per intermediate record of the run (sbp::get_intermediates): the reference's columns
  tag, numvertices, numedges, overlap, blocksizevar, undirected, algorithm, iteration, mdl,
  normalized_mdl_v1, normalized_mdl_v2, modularity, interblock_edges, block_size_variation,
  f1_score, nmi, true_mdl, true_mdl_v1, true_mdl_v2, runtime, mcmc_iterations
then num_blocks, visits, seconds (device seconds since the partition started), vertex_moves_per_s
(visits / seconds) and, when given, eval_kernel_gbps and eval_roofline_frac (the vertex-evaluation
kernel's algorithmic bytes over its time, and that over the HBM peak).  The file is appended to
and gets the header when it is created, as the reference does; the path is
<csv><numvertices>/<type>.csv as the reference builds it from its --csv and --type flags.
"""
import math
import os

COLUMNS = ["tag", "numvertices", "numedges", "overlap", "blocksizevar", "undirected", "algorithm", "iteration",
           "mdl", "normalized_mdl_v1", "normalized_mdl_v2", "modularity", "interblock_edges",
           "block_size_variation", "f1_score", "nmi", "true_mdl", "true_mdl_v1", "true_mdl_v2", "runtime",
           "mcmc_iterations", "num_blocks", "visits", "seconds", "vertex_moves_per_s", "eval_kernel_gbps",
           "eval_roofline_frac"]


def null_mdl_v1(E):
    """entropy::null_mdl_v1 (src/entropy.cpp:567-573)."""
    x = 1.0 / E
    return E * ((1 + x) * math.log(1 + x) - x * math.log(x)) - E * math.log(1.0 / E)


def null_mdl_v2(V, E):
    """entropy::null_mdl_v2 (src/entropy.cpp:575-583)."""
    x = V * V / E
    return E * ((1 + x) * math.log(1 + x) - x * math.log(x)) + V * math.log(V) - E * math.log(1.0 / E)


def results_path(csv_dir, num_vertices, graph_type):
    return os.path.join(f"{csv_dir}{num_vertices}", f"{graph_type}.csv")


def write_results(path, intermediates, *, num_vertices, num_edges, algorithm, evaluation, runtime, tag="default",
                  overlap="", blocksizevar="", undirected=False, eval_kernel_gbps=None, hbm_peak_gbps=None):
    """Append one row per intermediate record; `evaluation` is sbp_evaluate_blockmodel's result
    (f1_score, nmi, true_mdl) of the final partition, `runtime` its wall seconds."""
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    exists = os.path.exists(path)
    tm = evaluation.get("true_mdl", float("nan"))
    frac = (eval_kernel_gbps / hbm_peak_gbps) if (eval_kernel_gbps and hbm_peak_gbps) else None
    with open(path, "a") as f:
        if not exists:
            f.write(", ".join(COLUMNS) + "\n")
        for r in intermediates:
            row = [tag, num_vertices, num_edges, overlap, blocksizevar, int(bool(undirected)), algorithm,
                   r["iteration"], r["mdl"], r["normalized_mdl_v1"], r["normalized_mdl_v2"], r["modularity"],
                   r["interblock_edges"], r["block_size_variation"], evaluation["f1_score"], evaluation["nmi"], tm,
                   tm / null_mdl_v1(num_edges), tm / null_mdl_v2(num_vertices, num_edges), runtime,
                   r["mcmc_iterations"], r["num_blocks"], r["visits"], r["seconds"],
                   (r["visits"] / r["seconds"]) if r["seconds"] > 0 else 0.0,
                   "" if eval_kernel_gbps is None else eval_kernel_gbps, "" if frac is None else frac]
            f.write(", ".join(str(x) for x in row) + "\n")
    return path
