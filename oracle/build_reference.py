"""Build the reference (vtsynergy/Hybrid-Stochastic-Block-Partitioning) from its own sources.

TEST INFRASTRUCTURE ONLY.  The reference's sources stay where they lie; nothing is copied.  Its
build system (CMake with MPI, robin-map, abseil and googletest) is not used: its library
sources are compiled directly with g++ -O3 -fopenmp against the project-written shims in
oracle/ref_shims (single-process MPI, robin_map -> std::unordered_map, an empty abseil header,
missing standard includes), together with oracle/ref_driver.cpp.  Output: oracle/_ref/.

The built driver is the CPU baseline of bench.py (--impl reference and the cpu_baseline field).
"""
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("SBP_REFERENCE_DIR", "/root/reference")
OUT = os.path.join(HERE, "_ref")
DRIVER = os.path.join(OUT, "ref_driver")
SOURCES = [
    "src/graph.cpp", "src/utils.cpp", "src/sbp.cpp", "src/entropy.cpp", "src/evaluate.cpp", "src/common.cpp",
    "src/finetune.cpp", "src/block_merge.cpp", "src/partition.cpp", "src/blockmodel/blockmodel.cpp",
    "src/blockmodel/blockmodel_triplet.cpp", "src/blockmodel/dist_blockmodel.cpp",
    "src/blockmodel/sparse/dict_matrix.cpp", "src/blockmodel/sparse/dict_transpose_matrix.cpp",
    "extern/hungarian/hungarian.cpp",
]
INCLUDES = ["include", "include/blockmodel", "include/blockmodel/sparse", "patches", "extern/hungarian",
            "extern/tclap-1.2.2/include"]


def reference_available():
    return all(os.path.exists(os.path.join(REF, s)) for s in SOURCES)


def built():
    return os.path.exists(DRIVER)


def build(force=False, jobs=8):
    if built() and not force:
        return DRIVER
    if not reference_available():
        raise RuntimeError("reference sources not found")
    os.makedirs(os.path.join(OUT, "obj"), exist_ok=True)
    shims = os.path.join(HERE, "ref_shims")
    flags = ["-std=c++17", "-O3", "-fopenmp", "-w", "-I" + shims] + ["-I" + os.path.join(REF, i) for i in INCLUDES] + \
            ["-include", os.path.join(shims, "ref_prelude.h")]
    procs, objs = [], []
    for src in SOURCES + [os.path.join(HERE, "ref_driver.cpp")]:
        path = src if os.path.isabs(src) else os.path.join(REF, src)
        obj = os.path.join(OUT, "obj", os.path.basename(src).replace(".cpp", ".o"))
        objs.append(obj)
        procs.append(subprocess.Popen(["g++"] + flags + ["-c", path, "-o", obj]))
        if len(procs) >= jobs:
            if procs.pop(0).wait() != 0:
                raise RuntimeError("reference compile failed: " + src)
    for p in procs:
        if p.wait() != 0:
            raise RuntimeError("reference compile failed")
    subprocess.check_call(["g++", "-fopenmp", "-o", DRIVER] + objs)
    return DRIVER


def _write_edges(path, V, src, dst):
    with open(path, "wb") as f:
        f.write(np.int32(V).tobytes())
        f.write(np.int64(len(src)).tobytes())
        f.write(np.ascontiguousarray(src, np.int32).tobytes())
        f.write(np.ascontiguousarray(dst, np.int32).tobytes())


def run_finetune(V, src, dst, assignment, algo="async_gibbs", batches=10, threads=None):
    threads = threads or os.cpu_count()
    with tempfile.TemporaryDirectory() as d:
        e, a = os.path.join(d, "e.bin"), os.path.join(d, "a.bin")
        _write_edges(e, V, src, dst)
        with open(a, "wb") as f:
            f.write(np.int32(int(assignment.max()) + 1).tobytes())
            f.write(np.ascontiguousarray(assignment, np.int32).tobytes())
        out = subprocess.run([DRIVER, "finetune", e, algo, a, str(batches), str(threads)], capture_output=True,
                             text=True, check=True).stdout
    return json.loads(out.strip().splitlines()[-1])


def run_sbp(V, src, dst, algo="async_gibbs", batches=10, threads=None, approximate=True):
    threads = threads or os.cpu_count()
    with tempfile.TemporaryDirectory() as d:
        e, o = os.path.join(d, "e.bin"), os.path.join(d, "out.bin")
        _write_edges(e, V, src, dst)
        out = subprocess.run([DRIVER, "sbp", e, algo, str(batches), str(threads), str(int(approximate)), o],
                             capture_output=True, text=True, check=True).stdout
        raw = np.fromfile(o, dtype=np.int32)
    res = json.loads(out.strip().splitlines()[-1])
    res["assignment"] = raw[1:]
    return res


def split_blocks(truth, parts=10, seed=0):
    """The planted partition with every block split into `parts` random sub-blocks: a structured
    mid-range state (B = parts * K) like the ones the SBP search passes through."""
    rng = np.random.default_rng(seed)
    return (truth.astype(np.int64) * parts + rng.integers(0, parts, len(truth))).astype(np.int32)


def time_reference(V, src, dst, truth, budget_s=12.0, algo="async_gibbs", batches=10, parts=10):
    """Vertex visits/s of one reference finetune call on every host core, started from the
    planted partition split into `parts` sub-blocks per block (the bounded sample)."""
    a = split_blocks(truth, parts)
    r = run_finetune(V, src, dst, a, algo=algo, batches=batches)
    name = "asynchronous_gibbs" if algo == "async_gibbs" else algo
    return {"value": r["visits"] / r["seconds"], "unit": "vertex visits/s", "cores": r["threads"],
            "kind": "reference",
            "sample": f"one reference finetune::{name} call (batches {batches}, --transpose) from the planted "
                      f"partition split into {parts} sub-blocks per block (B={int(a.max()) + 1}) on the same graph: "
                      f"{r['sweeps']} sweeps, {r['visits']} visits in {r['seconds']:.2f} s"}


if __name__ == "__main__":
    t = time.time()
    print(build(force="--force" in sys.argv), f"{time.time() - t:.1f}s")
