"""Record the reference's full sbp::stochastic_block_partition on a benchmark graph: wall time
(time to final MDL), MCMC time and sweeps, final MDL and blocks, NMI against the planted
partition, and the host it ran on.  TEST INFRASTRUCTURE ONLY: the numbers go to
oracle/reference_anchors.json, which bench.py's reference arm carries beside its bounded sample.

Run:  python oracle/record_reference_anchor.py <config> [threads]
The reference is the unmodified build (oracle/_ref/ref_driver, oracle/build_reference.py).
"""
import json
import os
import platform
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "hybrid-stochastic-block-partitioning_b200"))

import build_reference as R  # noqa: E402
import dcsbm  # noqa: E402
import sbp_oracle as O  # noqa: E402

OUT = os.path.join(HERE, "reference_anchors.json")


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor()


def main(cfg, threads):
    R.build()
    V, s, d, truth = dcsbm.config_graph(cfg)
    t0 = time.time()
    res = R.run_sbp(V, s, d, algo="async_gibbs", batches=10, threads=threads)
    wall = time.time() - t0
    rec = {"algorithm": "async_gibbs", "batches": 10, "approximate": True, "threads": threads,
           "host_cores": os.cpu_count(), "cpu": cpu_model(), "partition_seconds": res["seconds"],
           "mcmc_seconds": res["mcmc_seconds"], "sweeps": res["sweeps"], "final_mdl": res["mdl"],
           "final_blocks": res["num_blocks"], "nmi_vs_planted": float(O.nmi(res["assignment"], truth)),
           "E": res["E"], "V": res["V"], "process_wall_seconds": wall}
    bs = -(-V // 10)   # asynchronous Gibbs visits (V / batch_size) * batch_size vertices per sweep
    rec["visits"] = res["sweeps"] * (V // bs) * bs
    rec["visits_per_mcmc_second"] = rec["visits"] / res["mcmc_seconds"]
    rec["visits_per_partition_second"] = rec["visits"] / res["seconds"]
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    data[str(cfg)] = rec
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1)
    print(json.dumps(rec))


if __name__ == "__main__":
    main(int(sys.argv[1]), int(sys.argv[2]) if len(sys.argv) > 2 else os.cpu_count())
