"""Runs the patched reference build (oracle/_ref/replay/ref_driver, made by
oracle/build_reference.py) and reads the log it writes.  TEST INFRASTRUCTURE ONLY.

The log holds every finetune and merge call of the run: the blockmodel state at its start and
at its end, and the random stream the reference drew in it: for each vertex visit the proposed
block and the accept uniform, for each merge proposal the proposed block.  `finetune_stream`
and `merge_stream` turn a call's records into the arrays the GPU engine's replay entry points
take (record t*V + v for the visit of vertex v in sweep t; record block*10 + i for merge
proposal i of a block).
"""
import json
import os
import subprocess
import tempfile

import numpy as np

import build_reference as R

KINDS = {0: "metropolis_hastings", 1: "async_gibbs", 2: "hybrid_mcmc", 3: "merge"}
PROPOSALS_PER_BLOCK = 10   # NUM_AGG_PROPOSALS_PER_BLOCK (include/block_merge.hpp)


class Reader:
    def __init__(self, data):
        self.d = data
        self.i = 0

    def take(self, dtype, n=1):
        a = np.frombuffer(self.d, dtype=dtype, count=n, offset=self.i)
        self.i += a.nbytes
        return a

    def i32(self):
        return int(self.take(np.int32)[0])

    def state(self):
        B, V, to_merge = (int(x) for x in self.take(np.int32, 3))
        entropy = float(self.take(np.float32)[0])
        b = self.take(np.int32, V).copy()
        d_out = self.take(np.int32, B).copy()
        d_in = self.take(np.int32, B).copy()
        d = self.take(np.int32, B).copy()
        nnz = int(self.take(np.int64)[0])
        cells = self.take(np.int32, 3 * nnz).reshape(nnz, 3).copy()
        return {"B": B, "V": V, "num_blocks_to_merge": to_merge, "overall_entropy": entropy, "assignment": b,
                "d_out": d_out, "d_in": d_in, "d": d, "cells": cells}


def matrix(state):
    """Dense B x B counts of a logged state."""
    M = np.zeros((state["B"], state["B"]), np.int32)
    c = state["cells"]
    M[c[:, 0], c[:, 1]] = c[:, 2]
    return M


def read_log(path):
    with open(path, "rb") as f:
        r = Reader(f.read())
    calls = {}
    order = []
    split = None
    while r.i < len(r.d):
        tag = r.d[r.i:r.i + 1]
        r.i += 1
        if tag == b"B":
            cid, kind, bracket = r.i32(), r.i32(), r.i32()
            calls[cid] = {"id": cid, "kind": KINDS[kind], "bracket": bracket, "begin": r.state(), "visits": [], "uniforms": [],
                          "merge": [], "scores": None}
            order.append(cid)
        elif tag == b"E":
            cid, kind, sweeps = r.i32(), r.i32(), r.i32()
            calls[cid]["sweeps"] = sweeps
            calls[cid]["end"] = r.state()
        elif tag == b"P":
            calls_rec = r.take(np.int32, 4)
            calls[int(calls_rec[0])]["visits"].append(calls_rec[1:].copy())
        elif tag == b"U":
            rec = r.take(np.int32, 3)
            u = float(r.take(np.float64)[0])
            calls[int(rec[0])]["uniforms"].append((int(rec[1]), int(rec[2]), u))
        elif tag == b"M":
            rec = r.take(np.int32, 4)
            calls[int(rec[0])]["merge"].append(rec[1:].copy())
        elif tag == b"S":
            cid, B = r.i32(), r.i32()
            best = r.take(np.int32, B).copy()
            delta = r.take(np.float64, B).copy()
            calls[cid]["scores"] = (best, delta)
        elif tag == b"G":
            high = r.take(np.int32, r.i32()).copy()
            low = r.take(np.int32, r.i32()).copy()
            split = (high, low)
        else:
            raise ValueError(f"bad replay log tag {tag!r} at byte {r.i - 1}")
    return [calls[c] for c in order], split


def finetune_stream(call, V):
    """(proposal[sweeps*V], uniform[sweeps*V]) of a logged finetune call; -1 / 2.0 where the
    reference made no such draw (a vertex it did not visit; a visit that kept its block)."""
    n = max(1, call["sweeps"]) * V
    prop = np.full(n, -1, np.int32)
    uni = np.full(n, 2.0, np.float64)
    if call["visits"]:
        v = np.array(call["visits"], np.int64)
        prop[v[:, 0] * V + v[:, 1]] = v[:, 2]
    for sweep, vertex, u in call["uniforms"]:
        uni[sweep * V + vertex] = u
    return prop, uni


def merge_stream(call):
    B = call["begin"]["B"]
    prop = np.full(B * PROPOSALS_PER_BLOCK, -1, np.int32)
    if call["merge"]:
        m = np.array(call["merge"], np.int64)
        prop[m[:, 0] * PROPOSALS_PER_BLOCK + m[:, 1]] = m[:, 2]
    return prop


def _env(log, seed, max_sweeps):
    env = dict(os.environ)
    env["SBP_REPLAY_LOG"] = log
    env["SBP_REF_SEED"] = str(seed)
    env["SBP_REF_MAX_SWEEPS"] = str(max_sweeps)
    return env


def run(mode, V, src, dst, *, algo="async_gibbs", assignment=None, batches=10, threads=None, approximate=True,
        num_blocks_to_merge=0, seed=1, max_sweeps=100):
    """Run the patched reference once (mode "sbp", "finetune" or "merge") and return
    (driver JSON line, logged calls)."""
    if not R.replay_built():
        R.build_replay()
    threads = threads or os.cpu_count()
    with tempfile.TemporaryDirectory() as d:
        e, a, o, log = (os.path.join(d, x) for x in ("e.bin", "a.bin", "o.bin", "replay.log"))
        R._write_edges(e, V, src, dst)
        if assignment is not None:
            with open(a, "wb") as f:
                f.write(np.int32(int(assignment.max()) + 1).tobytes())
                f.write(np.ascontiguousarray(assignment, np.int32).tobytes())
        if mode == "sbp":
            cmd = [R.REPLAY_DRIVER, "sbp", e, algo, str(batches), str(threads), str(int(approximate)), o]
        elif mode == "finetune":
            cmd = [R.REPLAY_DRIVER, "finetune", e, algo, a, str(batches), str(threads)]
        else:
            cmd = [R.REPLAY_DRIVER, "merge", e, a, str(num_blocks_to_merge), str(threads), str(int(approximate))]
        out = subprocess.run(cmd, capture_output=True, text=True, check=True, env=_env(log, seed, max_sweeps)).stdout
        res = json.loads(out.strip().splitlines()[-1])
        if mode == "sbp":
            res["assignment"] = np.fromfile(o, dtype=np.int32)[1:]
        calls, split = read_log(log)
        res["split"] = split
        return res, calls
