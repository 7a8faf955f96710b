"""Seeded directed degree-corrected SBM generator for the benchmark and test graphs.

The reference's own generator (SBMGraphGenerator/generate.py, graph-tool based) is not in the
reference repository, so this is a project-written stand-in with the law its wrapper script
describes (SBMGraphGenerator/generate_graphs.sh: power-law degrees, within-block fraction,
block-size variation):
  * block proportions ~ Dirichlet(alpha) (alpha = 10 for "low" variation, 1 for "high"),
    every block non-empty;
  * out-degree of each vertex ~ discrete power law p(k) ~ k^-gamma on [k_min, k_max];
  * each out-edge stays in the source's block with probability w, otherwise it may land in
    any block; the target is drawn proportionally to a per-vertex popularity (same power law),
    which gives the in-degree correction;
  * vertex ids are shuffled; duplicate edges are left in the list (the graph loader drops
    them, as Graph::load_text does) and self loops may occur.
Everything is a function of the seed.
"""
import math
import os

import numpy as np

# The suite's graphs by suite number (seeds fixed; the batched suite is batched_config):
#   1  1,000 vertices, 11 blocks, low size variation: the small plain-SBP case the reference runs in seconds
#   2  20,000 vertices, 32 blocks, high variation and overlap: asynchronous Gibbs, hybrid, replay at scale
#   4  200,000 vertices, 71 blocks: the bench graph (vertex moves/s, learned vs plain proposal)
#   5  2,000,000 vertices, 150 blocks, degree exponent 2.1 on [10, 200]: the large hybrid case
CONFIGS = {
    1: dict(V=1_000, K=11, alpha=10.0, gamma=2.5, kmin=10, kmax=100, w=0.8, seed=1),
    2: dict(V=20_000, K=32, alpha=1.0, gamma=2.5, kmin=10, kmax=100, w=0.6, seed=2),
    4: dict(V=200_000, K=71, alpha=1.0, gamma=2.5, kmin=10, kmax=100, w=0.7, seed=4),
    5: dict(V=2_000_000, K=150, alpha=10.0, gamma=2.1, kmin=10, kmax=200, w=0.75, seed=5),
}


def batched_config(g):
    """Graph g (0..63) of the batched suite: V log-uniform in [1k, 50k], K = round(1.2 V^0.35)."""
    rng = np.random.default_rng(3 + g)
    V = int(round(math.exp(rng.uniform(math.log(1_000), math.log(50_000)))))
    return dict(V=V, K=int(round(1.2 * V ** 0.35)), alpha=3.0, gamma=2.5, kmin=10, kmax=100,
                w=float(rng.uniform(0.5, 0.9)), seed=3 + g)


def _power_law(rng, n, gamma, kmin, kmax):
    k = np.arange(kmin, kmax + 1, dtype=np.float64)
    p = k ** (-gamma)
    cdf = np.cumsum(p / p.sum())
    return (kmin + np.searchsorted(cdf, rng.random(n), side="right")).astype(np.int64).clip(kmin, kmax)


def generate(V, K, alpha, gamma, kmin, kmax, w, seed):
    """Return (V, src, dst, truth) with int32 arrays; truth is the planted block of each vertex."""
    rng = np.random.default_rng(seed)
    props = rng.dirichlet(np.full(K, alpha))
    sizes = 1 + rng.multinomial(V - K, props)
    block_of = np.repeat(np.arange(K), sizes)
    perm = rng.permutation(V)               # vertex id -> position in block order
    truth = np.empty(V, np.int64)
    truth[perm] = block_of                  # vertex perm[i] gets block_of[i]
    members = [perm[np.arange(sizes[:b].sum(), sizes[:b + 1].sum())] for b in range(K)]
    theta = _power_law(rng, V, gamma, kmin, kmax).astype(np.float64)
    deg = _power_law(rng, V, gamma, kmin, kmax)
    src = np.repeat(np.arange(V, dtype=np.int64), deg)
    within = rng.random(len(src)) < w
    dst = np.empty(len(src), np.int64)
    # within-block targets, popularity-weighted inside the source's block
    sb = truth[src]
    for b in range(K):
        sel = np.nonzero(within & (sb == b))[0]
        if len(sel) == 0:
            continue
        m = members[b]
        cdf = np.cumsum(theta[m])
        cdf /= cdf[-1]
        dst[sel] = m[np.minimum(np.searchsorted(cdf, rng.random(len(sel)), side="right"), len(m) - 1)]
    # cross-block targets, popularity-weighted over all vertices
    sel = np.nonzero(~within)[0]
    cdf = np.cumsum(theta)
    cdf /= cdf[-1]
    dst[sel] = np.minimum(np.searchsorted(cdf, rng.random(len(sel)), side="right"), V - 1)
    return V, src.astype(np.int32), dst.astype(np.int32), truth.astype(np.int32)


def config_graph(cfg):
    c = CONFIGS[cfg] if isinstance(cfg, int) else cfg
    return generate(**c)


def write_tsv(path_base, src, dst, truth):
    """Write `<base>.tsv` (1-indexed "from\\tto") and `<base>_truePartition.tsv` in the layout
    the reference's loader reads (src/graph.cpp:24-63, src/utils.cpp:19-42)."""
    os.makedirs(os.path.dirname(path_base) or ".", exist_ok=True)
    np.savetxt(path_base + ".tsv", np.stack([src + 1, dst + 1], 1), fmt="%d", delimiter="\t")
    np.savetxt(path_base + "_truePartition.tsv", np.stack([np.arange(len(truth)) + 1, truth + 1], 1), fmt="%d",
               delimiter="\t")
