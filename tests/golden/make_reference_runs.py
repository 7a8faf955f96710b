"""Run the reference (built from its sources by oracle/build_reference.py) end to end on the
benchmark graphs and record its final MDL, number of blocks and NMI to the planted partition
in reference_runs.json.  The reference draws from an unseeded std::random_device, so each
record is one sample of its output; the GPU engine is checked against these within the
end-to-end tolerance (final MDL within 0.5 %, NMI within 0.01).
Run:  python tests/golden/make_reference_runs.py [config ...]
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "hybrid-stochastic-block-partitioning_b200"))
import build_reference as R  # noqa: E402
import dcsbm  # noqa: E402
import sbp_oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_runs.json")


def main(configs):
    R.build()
    runs = json.load(open(OUT)) if os.path.exists(OUT) else []
    for cfg in configs:
        V, s, d, truth = dcsbm.config_graph(cfg)
        for algo in ("metropolis_hastings", "async_gibbs", "hybrid_mcmc"):
            if any(r["config"] == cfg and r["algorithm"] == algo for r in runs):
                continue
            r = R.run_sbp(V, s, d, algo=algo, batches=10, approximate=True)
            a = r.pop("assignment")
            r.update(config=cfg, algorithm=algo, batches=10, approximate=True, nmi=O.nmi(a, truth))
            runs.append(r)
            json.dump(runs, open(OUT, "w"), indent=1)
            print(r, flush=True)


if __name__ == "__main__":
    main([int(c) for c in sys.argv[1:]] or [1])
