"""Build the reference (vtsynergy/Hybrid-Stochastic-Block-Partitioning) from its own sources.

TEST INFRASTRUCTURE ONLY.  Its build system (CMake with MPI, robin-map, abseil and googletest) is
not used: its library sources are compiled directly with g++ -O3 -fopenmp against the project-
written shims in oracle/ref_shims (single-process MPI, robin_map -> std::unordered_map, an empty
abseil header, missing standard includes), together with oracle/ref_driver.cpp.

Two builds, both under oracle/_ref/ (git-ignored; nothing from the reference is committed):
  * oracle/_ref/ref_driver: the unmodified sources where they lie.  The CPU baseline of
    bench.py (--impl reference and the cpu_baseline field) and the unseeded end-to-end runs.
  * oracle/_ref/replay/ref_driver: a copy of src/ and include/ under oracle/_ref/replay/ with
    the patches of REPLAY_PATCHES applied (seeded engines and a log of every proposal and accept
    uniform, FP64 logs, a fixed tie order of merges, a sweep cap) and the hooks of
    oracle/ref_replay/sbp_replay.cpp.  The seeded-replay parity tests run the GPU engine on the
    stream this build logs and compare every finetune and merge call's end state with it.
"""
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference checkout: SBP_REFERENCE_DIR, else a sibling `reference` directory of the repo's
# parent (where the build container mounts it).  Not needed on a machine that only runs the
# prebuilt oracle/_ref binaries.
REF = os.environ.get("SBP_REFERENCE_DIR") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
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


def _compile(root, out_dir, driver, extra_sources=(), extra_flags=(), jobs=8, driver_main=True, link=()):
    """Compile the reference's library sources under `root` (plus the project's driver, unless
    driver_main is false, and `extra_sources`) into `driver`."""
    os.makedirs(os.path.join(out_dir, "obj"), exist_ok=True)
    shims = os.path.join(HERE, "ref_shims")
    incs = [os.path.join(root, i) for i in INCLUDES if os.path.isdir(os.path.join(root, i))] + \
           [os.path.join(REF, i) for i in INCLUDES]
    flags = ["-std=c++17", "-O3", "-fopenmp", "-w", "-I" + shims, "-I" + HERE] + ["-I" + i for i in incs] + \
            ["-include", os.path.join(shims, "ref_prelude.h")] + list(extra_flags)
    procs, objs = [], []
    srcs = [os.path.join(root if os.path.exists(os.path.join(root, s)) else REF, s) for s in SOURCES]
    mains = [os.path.join(HERE, "ref_driver.cpp")] if driver_main else []
    for path in srcs + mains + list(extra_sources):
        obj = os.path.join(out_dir, "obj", os.path.basename(path).replace(".cpp", ".o"))
        objs.append(obj)
        procs.append((path, subprocess.Popen(["g++"] + flags + ["-c", path, "-o", obj])))
        if len(procs) >= jobs:
            path0, p0 = procs.pop(0)
            if p0.wait() != 0:
                raise RuntimeError("reference compile failed: " + path0)
    for path0, p0 in procs:
        if p0.wait() != 0:
            raise RuntimeError("reference compile failed: " + path0)
    subprocess.check_call(["g++", "-fopenmp", "-o", driver] + objs + list(link))
    return driver


def build(force=False, jobs=8):
    if built() and not force:
        return DRIVER
    if not reference_available():
        raise RuntimeError("reference sources not found")
    return _compile(REF, OUT, DRIVER, jobs=jobs)


# ---- the reference-facing C++ adapter, built into a program of the reference's own classes ----------
ROOT = os.path.dirname(HERE)
PKG = os.path.join(ROOT, "hybrid-stochastic-block-partitioning_b200")
ADAPTER_OUT = os.path.join(OUT, "adapter")
ADAPTER_CHECK = os.path.join(ADAPTER_OUT, "adapter_check")


def adapter_built():
    return os.path.exists(ADAPTER_CHECK)


def build_adapter_check(force=False, jobs=8):
    """oracle/adapter_check.cpp + include/sbp_b200_reference.hpp against the reference's headers and
    library sources, linked with libsbp_b200.so (found at run time relative to the program)."""
    if adapter_built() and not force:
        return ADAPTER_CHECK
    if not reference_available():
        raise RuntimeError("reference sources not found")
    lib = os.path.join(PKG, "libsbp_b200.so")
    if not os.path.exists(lib):
        raise RuntimeError("libsbp_b200.so is not built")
    rpath = "$ORIGIN/" + os.path.relpath(PKG, ADAPTER_OUT)
    return _compile(REF, ADAPTER_OUT, ADAPTER_CHECK, extra_sources=[os.path.join(HERE, "adapter_check.cpp")],
                    extra_flags=["-I" + os.path.join(ROOT, "include"), "-I" + HERE], jobs=jobs, driver_main=False,
                    link=["-L" + PKG, "-lsbp_b200", "-Wl,-rpath," + rpath])


# ---- the replay build -------------------------------------------------------------------------
REPLAY_OUT = os.path.join(OUT, "replay")
REPLAY_DRIVER = os.path.join(REPLAY_OUT, "ref_driver")
HOOKS = os.path.join(HERE, "ref_replay")
_FT_PROPOSAL = r"(utils::ProposalAndEdgeCounts proposal = common::propose_new_block\([^;]*\);)"
_MERGE_PROPOSAL = "common::propose_new_block(current_block, out_blocks, in_blocks, block_assignment, blockmodel, true);"

# (file, kind, anchor, replacement, expected count).  kind: "lit" replaces every occurrence of a
# literal (exactly `count` of them), "first" only the first, "re" a regular expression, "after"
# the first occurrence of the anchor's second part that follows its first part.
REPLAY_PATCHES = [
    # P1: seeded per-translation-unit engines (include/common.hpp:25-26)
    ("include/common.hpp", "lit", "static std::random_device seeder;\nstatic std::default_random_engine generator(seeder());",
     "static std::default_random_engine generator(sbp_replay::seed());", 1),
    # P2: FP64 cell entropy (include/common.hpp:35-44) and nat_log (include/utils.hpp:145-151)
    ("include/common.hpp", "lit",
     "inline float cell_entropy(float value, float degree_in, float degree_out) {\n    if (value == 0.0) return 0.0;\n"
     "    float entropy = value * logf(value / (degree_in * degree_out));",
     "inline double cell_entropy(double value, double degree_in, double degree_out) {\n    if (value == 0.0) return 0.0;\n"
     "    double entropy = value * log(value / (degree_in * degree_out));", 1),
    ("include/utils.hpp", "lit", "result.push_back(logf(value));", "result.push_back(log(value));", 1),
    # P4: sweep cap of the finetune loops (include/finetune.hpp:56)
    ("include/finetune.hpp", "lit", "static const int MAX_NUM_ITERATIONS = 100;",
     "static const int MAX_NUM_ITERATIONS = sbp_replay::max_sweeps();", 1),
    # P1: accept uniform (src/finetune.cpp:22), visit proposals (:494, :510, :538), call records
    ("src/finetune.cpp", "lit", "double random_probability = distribution(common::generator);",
     "double random_probability = distribution(common::generator);\n    sbp_replay::on_uniform(random_probability);", 1),
    ("src/finetune.cpp", "re", _FT_PROPOSAL, r"\1\n    sbp_replay::on_proposal(vertex, proposal.proposal);", 3),
    ("src/finetune.cpp", "lit", 'std::cout << "Asynchronous Gibbs iteration" << std::endl;',
     'std::cout << "Asynchronous Gibbs iteration" << std::endl;\n'
     "    sbp_replay::CallScope sbp_replay_call(sbp_replay::kAsyncGibbs, blockmodel, blockmodels.get(2).empty ? 0 : 1);", 1),
    ("src/finetune.cpp", "lit", 'std::cout << "Hybrid MCMC iteration" << std::endl;',
     'std::cout << "Hybrid MCMC iteration" << std::endl;\n'
     "    sbp_replay::CallScope sbp_replay_call(sbp_replay::kHybrid, blockmodel, blockmodels.get(2).empty ? 0 : 1);", 1),
    ("src/finetune.cpp", "lit", 'std::cout << "Metropolis hastings iteration" << std::endl;',
     'std::cout << "Metropolis hastings iteration" << std::endl;\n'
     "    sbp_replay::CallScope sbp_replay_call(sbp_replay::kMetropolisHastings, blockmodel, blockmodels.get(2).empty ? 0 : 1);", 1),
    # P1: merge call, proposal slots and records, per-block scores (src/block_merge.cpp:278-304, 335-345)
    ("src/block_merge.cpp", "lit", "Blockmodel &merge_blocks(Blockmodel &blockmodel, const Graph &graph, int num_edges) {",
     "Blockmodel &merge_blocks(Blockmodel &blockmodel, const Graph &graph, int num_edges) {\n"
     "    sbp_replay::CallScope sbp_replay_call(sbp_replay::kMerge, blockmodel);", 1),
    ("src/block_merge.cpp", "first", "for (int i = 0; i < NUM_AGG_PROPOSALS_PER_BLOCK; ++i) {",
     "for (int i = 0; i < NUM_AGG_PROPOSALS_PER_BLOCK; ++i) {\n            sbp_replay::on_merge_slot(current_block, i);", 1),
    ("src/block_merge.cpp", "first", '    std::cout << "Avoided " << num_avoided',
     "    sbp_replay::on_merge_scores(best_merge_for_each_block, delta_entropy_for_each_block);\n"
     '    std::cout << "Avoided " << num_avoided', 1),
    ("src/block_merge.cpp", "after", ("ProposalEvaluation propose_merge_sparse(int current_block", _MERGE_PROPOSAL),
     _MERGE_PROPOSAL + "\n    sbp_replay::on_merge_proposal(proposal.proposal);", 1),
    # P3: merge delta in one orientation (src/block_merge.cpp:342-345) and stable tie order
    # (src/blockmodel/blockmodel.cpp:52)
    ("src/block_merge.cpp", "after", ("ProposalEvaluation propose_merge_sparse(int current_block",
                                      "    Delta delta = blockmodel_delta(current_block, proposal.proposal, blockmodel);\n"
                                      "    //==========NEW==============\n"
                                      "    double delta_entropy = entropy::block_merge_delta_mdl(current_block, proposal, "
                                      "blockmodel, delta);"),
     "    double delta_entropy = sbp_replay::merge_delta_canonical(current_block, proposal.proposal,\n"
     "        proposal.num_out_neighbor_edges, proposal.num_in_neighbor_edges, blockmodel);", 1),
    ("src/blockmodel/blockmodel.cpp", "lit", "std::vector<int> best_merges = utils::sort_indices(delta_entropy_for_each_block);",
     "std::vector<int> best_merges = sbp_replay::stable_sort_indices(delta_entropy_for_each_block);", 1),
    # P3, advanced carry-out (src/block_merge.cpp:123-217): the priority queue breaks equal
    # delta-MDLs by block id (std::priority_queue leaves their order to its heap), and a queued
    # merge is re-evaluated as the canonical rounded score, as merges are ranked everywhere
    # (both anchors start at a line break: the file keeps a commented-out copy of the function)
    ("src/block_merge.cpp", "after", ("\nvoid carry_out_best_merges_advanced(",
                                      "\n    auto cmp_fxn = [](merge_t left, merge_t right) { return std::get<2>(left) > "
                                      "std::get<2>(right); };"),
     "\n    auto cmp_fxn = [](merge_t left, merge_t right) {\n"
     "        return std::get<2>(left) != std::get<2>(right) ? std::get<2>(left) > std::get<2>(right)\n"
     "                                                       : std::get<0>(left) > std::get<0>(right);\n"
     "    };", 1),
    ("src/block_merge.cpp", "lit",
     "double delta_entropy_actual = entropy::block_merge_delta_mdl(merge_from, proposal, blockmodel, delta);",
     "double delta_entropy_actual = sbp_replay::merge_delta_canonical(merge_from, merge_to, k_out, k_in, blockmodel);",
     1),
]


def _apply(text, kind, anchor, repl, count, name):
    import re
    if kind == "lit":
        n = text.count(anchor)
        if n != count:
            raise RuntimeError(f"replay patch anchor found {n}x (want {count}) in {name}: {anchor[:60]!r}")
        return text.replace(anchor, repl)
    if kind == "first":
        if anchor not in text:
            raise RuntimeError(f"replay patch anchor missing in {name}: {anchor[:60]!r}")
        return text.replace(anchor, repl, 1)
    if kind == "re":
        new, n = re.subn(anchor, repl, text)
        if n != count:
            raise RuntimeError(f"replay patch pattern matched {n}x (want {count}) in {name}: {anchor[:60]!r}")
        return new
    if kind == "after":
        head, target = anchor
        i = text.find(head)
        j = text.find(target, i) if i >= 0 else -1
        if j < 0:
            raise RuntimeError(f"replay patch anchor missing in {name}: {target[:60]!r}")
        return text[:j] + repl + text[j + len(target):]
    raise ValueError(kind)


def _fingerprint(patches, files):
    """Hash of a patched build's inputs that live in this repository (its patch list, hooks,
    driver and shims), so that a build made from older inputs counts as not built."""
    import hashlib
    h = hashlib.sha256(repr(patches).encode())
    for path in sorted(files):
        with open(path, "rb") as f:
            h.update(os.path.relpath(path, HERE).encode() + f.read())
    return h.hexdigest()


def _built_from(driver, out_dir, fingerprint):
    stamp = os.path.join(out_dir, "inputs.sha256")
    if not (os.path.exists(driver) and os.path.exists(stamp)):
        return False
    with open(stamp) as f:
        return f.read().strip() == fingerprint


def _stamp(out_dir, fingerprint):
    with open(os.path.join(out_dir, "inputs.sha256"), "w") as f:
        f.write(fingerprint + "\n")


def _files_under(d):
    return [os.path.join(r, n) for r, _, names in os.walk(d) for n in names if not n.endswith(".pyc")]


def _shim_files():
    return _files_under(os.path.join(HERE, "ref_shims")) + [os.path.join(HERE, "ref_driver.cpp")]


def _replay_fingerprint():
    return _fingerprint(REPLAY_PATCHES, _shim_files() + _files_under(HOOKS))


def replay_built():
    return _built_from(REPLAY_DRIVER, REPLAY_OUT, _replay_fingerprint())


def _patched_tree(out_dir, patches):
    """A copy of the reference's src/ and include/ under out_dir/tree with `patches` applied."""
    import shutil
    root = os.path.join(out_dir, "tree")
    if os.path.isdir(root):
        shutil.rmtree(root)
    for d in ("src", "include"):
        shutil.copytree(os.path.join(REF, d), os.path.join(root, d))
    for rel, kind, anchor, repl, count in patches:
        path = os.path.join(root, rel)
        with open(path) as f:
            text = f.read()
        text = _apply(text, kind, anchor, repl, count, rel)
        with open(path, "w") as f:
            f.write(text)
    return root


def build_replay(force=False, jobs=8):
    """Copy the reference's src/ and include/ to oracle/_ref/replay/, apply REPLAY_PATCHES and
    build the replay driver with the hooks of oracle/ref_replay."""
    if replay_built() and not force:
        return REPLAY_DRIVER
    if not reference_available():
        raise RuntimeError("reference sources not found")
    root = _patched_tree(REPLAY_OUT, REPLAY_PATCHES)
    out = _compile(root, REPLAY_OUT, REPLAY_DRIVER, extra_sources=[os.path.join(HOOKS, "sbp_replay.cpp")],
                   extra_flags=["-I" + HOOKS, "-include", os.path.join(HOOKS, "sbp_replay.h")], jobs=jobs)
    _stamp(REPLAY_OUT, _replay_fingerprint())
    return out


# ---- the capped timing build: the reference unchanged except for a sweep cap -------------------
# Bounded CPU-baseline samples need finetune calls of a few sweeps; MAX_NUM_ITERATIONS is a
# compile-time 100 (include/finetune.hpp:56).  Only that bound changes (SBP_REF_MAX_SWEEPS, default
# 100); FP32 logs, unseeded engines and everything else stay the reference's.
CAPPED_OUT = os.path.join(OUT, "capped")
CAPPED_DRIVER = os.path.join(CAPPED_OUT, "ref_driver")
CAPPED_PATCHES = [
    ("include/finetune.hpp", "lit", "static const int MAX_NUM_ITERATIONS = 100;",
     "static const int MAX_NUM_ITERATIONS = sbp_ref_sweep_cap();", 1),
]


def capped_built():
    return _built_from(CAPPED_DRIVER, CAPPED_OUT, _fingerprint(CAPPED_PATCHES, _shim_files()))


def build_capped(force=False, jobs=8):
    if capped_built() and not force:
        return CAPPED_DRIVER
    if not reference_available():
        raise RuntimeError("reference sources not found")
    root = _patched_tree(CAPPED_OUT, CAPPED_PATCHES)
    out = _compile(root, CAPPED_OUT, CAPPED_DRIVER,
                   extra_flags=["-include", os.path.join(HERE, "ref_shims", "sweep_cap.h")], jobs=jobs)
    _stamp(CAPPED_OUT, _fingerprint(CAPPED_PATCHES, _shim_files()))
    return out


def _write_edges(path, V, src, dst):
    with open(path, "wb") as f:
        f.write(np.int32(V).tobytes())
        f.write(np.int64(len(src)).tobytes())
        f.write(np.ascontiguousarray(src, np.int32).tobytes())
        f.write(np.ascontiguousarray(dst, np.int32).tobytes())


def run_finetune(V, src, dst, assignment, algo="async_gibbs", batches=10, threads=None, driver=None, max_sweeps=0):
    """One reference finetune call from `assignment` (labels 0..B-1, every block non-empty);
    max_sweeps > 0 caps the call's sweeps (the capped build)."""
    threads = threads or os.cpu_count()
    env = dict(os.environ)
    if max_sweeps > 0:
        driver = driver or CAPPED_DRIVER
        env["SBP_REF_MAX_SWEEPS"] = str(max_sweeps)
    with tempfile.TemporaryDirectory() as d:
        e, a = os.path.join(d, "e.bin"), os.path.join(d, "a.bin")
        _write_edges(e, V, src, dst)
        with open(a, "wb") as f:
            f.write(np.int32(int(assignment.max()) + 1).tobytes())
            f.write(np.ascontiguousarray(assignment, np.int32).tobytes())
        out = subprocess.run([driver or DRIVER, "finetune", e, algo, a, str(batches), str(threads)],
                             capture_output=True, text=True, check=True, env=env).stdout
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
    """The planted partition with every block split into `parts` random sub-blocks, relabelled
    0..B-1 (no empty block): a structured state with B near parts x planted blocks, like the
    ones the SBP search passes through."""
    rng = np.random.default_rng(seed)
    a = truth.astype(np.int64) * parts + rng.integers(0, parts, len(truth))
    _, a = np.unique(a, return_inverse=True)
    return a.astype(np.int32)


def halving_levels(V, K):
    """Block counts of sbp::stochastic_block_partition's first descent: V/2, V/4, ... while above
    the planted K, then K (the merges halve B each round, src/sbp.cpp:61-98)."""
    levels, B = [], V // 2
    while B > K:
        levels.append(B)
        B //= 2
    return levels + [K]


def spread_order(n):
    """0..n-1 in van der Corput order (0, n/2, n/4, 3n/4, ...): every prefix samples the whole
    range evenly, so a sample of the halving levels cut short by a time budget is not biased
    towards the largest or the smallest block counts."""
    out, seen = [], set()
    bits = max(1, (n - 1).bit_length())
    for i in range(1 << bits):
        j = int(format(i, f"0{bits}b")[::-1], 2)
        if j < n and j not in seen:
            seen.add(j)
            out.append(j)
    return out


def time_reference_level(V, src, dst, truth, B, batches=10, threads=None, algo="async_gibbs"):
    """One capped (1-sweep) reference finetune call at about B blocks: the planted partition split
    into B / K sub-blocks per block."""
    K = int(truth.max()) + 1
    a = split_blocks(truth, max(1, B // K), seed=B)
    r = run_finetune(V, src, dst, a, algo=algo, batches=batches, threads=threads, max_sweeps=1)
    r["B"] = int(a.max()) + 1
    return r


def time_reference(V, src, dst, truth, budget_s=20.0, batches=10, threads=None):
    """Vertex visits/s of the reference's asynchronous Gibbs on every host core, over 1-sweep
    calls at the partition's block-count levels (halving_levels) in spread order, until
    `budget_s` of sweep time: the bounded CPU baseline.  Every level of the partition's first
    descent runs the same number of sweeps, so visits over seconds across evenly spread levels
    estimates the whole descent's rate."""
    K = int(truth.max()) + 1
    all_levels = halving_levels(V, K)
    levels = [all_levels[i] for i in spread_order(len(all_levels))]
    visits, secs, done = 0, 0.0, []
    for B in levels:
        r = time_reference_level(V, src, dst, truth, B, batches, threads)
        visits += r["visits"]
        secs += r["seconds"]
        done.append(r["B"])
        if secs >= budget_s:
            break
    return {"value": visits / secs, "unit": "vertex visits/s", "cores": threads or os.cpu_count(), "kind": "reference",
            "sample": f"reference finetune::asynchronous_gibbs (batches {batches}, --transpose; the build's only change "
                      f"is a sweep cap) for 1 sweep at each of B = {done} (the planted partition split into B/K "
                      f"sub-blocks; levels of the partition's halving schedule in spread order): {visits} visits "
                      f"in {secs:.2f} s"}


if __name__ == "__main__":
    t = time.time()
    print(build(force="--force" in sys.argv), f"{time.time() - t:.1f}s")
