"""The reference-facing C++ adapter (include/sbp_b200_reference.hpp).

oracle/adapter_check.cpp is built against the reference's own headers and its Graph /
Blockmodel sources (oracle/build_reference.py) and calls sbp_b200::finetune::asynchronous_gibbs,
block_merge::merge_blocks, finetune::hybrid_mcmc, sbp::stochastic_block_partition and
entropy::mdl on the reference's own Blockmodel objects, then reads them back through the
reference's accessors (blockmatrix()->get, degrees_out / degrees_in / degrees).

CPU: the program builds and links the library, and without a device every call reports the
engine's no-device error (SBP_ERR_CUDA) instead of falling back to the CPU.
GPU: every step's state equals the ctypes path's (same seeds, same call words) bit for bit.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import random_graph


def adapter():
    import build_reference as R
    if not R.adapter_built():
        if not R.reference_available():
            pytest.fail("oracle/_ref/adapter/adapter_check is not built and the reference sources are absent")
        R.build_adapter_check()
    return R


def run_adapter(V, src, dst, B, assignment, seed):
    R = adapter()
    with tempfile.TemporaryDirectory() as td:
        e, a, o = (os.path.join(td, x) for x in ("e.bin", "a.bin", "o.bin"))
        R._write_edges(e, V, src, dst)
        with open(a, "wb") as f:
            f.write(np.int32(B).tobytes())
            f.write(np.ascontiguousarray(assignment, np.int32).tobytes())
        r = subprocess.run([R.ADAPTER_CHECK, e, a, o, str(seed)], capture_output=True, text=True)
        raw = np.fromfile(o, dtype=np.uint8) if os.path.exists(o) else np.zeros(0, np.uint8)
    return r, raw.tobytes()


def parse(raw, V):
    pos = 0

    def ints(n):
        nonlocal pos
        a = np.frombuffer(raw, np.int32, n, pos).copy()
        pos += 4 * n
        return a

    high = ints(int(ints(1)[0]))
    low = ints(int(ints(1)[0]))
    steps = []
    while pos < len(raw):
        B, VV = (int(x) for x in ints(2))
        assert VV == V
        st = {"B": B, "b": ints(V), "d_out": ints(B), "d_in": ints(B), "d": ints(B), "M": ints(B * B).reshape(B, B)}
        st["mdl"] = float(np.frombuffer(raw, np.float64, 1, pos)[0])
        pos += 8
        steps.append(st)
    return (high, low), steps


def small_case():
    V, s, d, _ = random_graph(300, 6, 11, kmax=30, w=0.8)
    a = (np.arange(V) % 12).astype(np.int32)
    return V, s, d, 12, a


def test_adapter_builds_and_reports_no_device_without_a_gpu():
    import sbp_b200 as S
    S.load()
    if S.device_count() > 0:
        pytest.skip("a CUDA device is present: the GPU test covers the adapter")
    V, s, d, B, a = small_case()
    r, _ = run_adapter(V, s, d, B, a, seed=5)
    assert r.returncode == 3, (r.stdout, r.stderr)
    assert "no CUDA device" in r.stdout


@pytest.mark.gpu
def test_adapter_matches_the_ctypes_path(S, O):
    V, s, d, B, a = small_case()
    seed = 5
    r, raw = run_adapter(V, s, d, B, a, seed)
    assert r.returncode == 0, (r.stdout, r.stderr)
    (high, low), steps = parse(raw, V)
    assert len(steps) == 4
    g = S.Graph(V, s, d)
    g.set_split(high, low)   # the reference's order of equal degrees, as the adapter passes it
    bm = S.Blockmodel(g, B, a)
    expect = []
    S.finetune.asynchronous_gibbs(bm, batches=10, seed=seed, call=0)
    expect.append(bm.copy())
    bm.setNum_blocks_to_merge(bm.B // 2)
    S.block_merge.merge_blocks(bm, approximate=True, seed=seed, call=1)
    expect.append(bm.copy())
    S.finetune.hybrid_mcmc(bm, batches=10, seed=seed, call=2)
    expect.append(bm.copy())
    out, st = S.sbp.stochastic_block_partition(g, batches=10, seed=seed)
    expect.append(S.Blockmodel(g, st["num_blocks"], out))
    og = O.Graph(V, s, d)
    for k, (e, got) in enumerate(zip(expect, steps)):
        assert got["B"] == e.B, k
        assert np.array_equal(got["b"], e.block_assignment()), k
        assert np.array_equal(got["M"], e.blockmatrix()), k
        do, di, dd = e.degrees_all()
        assert np.array_equal(got["d_out"], do) and np.array_equal(got["d_in"], di), k
        assert np.array_equal(got["d"], dd), k
        ref = O.Blockmodel(og, got["B"], got["b"]).mdl()
        assert got["mdl"] == pytest.approx(ref, rel=1e-9), k
