"""CPU tests of the product library without running kernels: it loads, exports every symbol
the C header declares, and refuses to compute (no CPU fallback) when no device is present."""
import os
import re

import numpy as np
import pytest

from conftest import PKG, ROOT


def header_symbols():
    text = open(os.path.join(ROOT, "include", "sbp_b200.h")).read()
    return sorted(set(re.findall(r"\b(sbp_[a-z_]+)\s*\(", text)))


def test_library_exports_header_symbols():
    import sbp_b200
    L = sbp_b200.load()
    syms = header_symbols()
    assert len(syms) >= 20
    for name in syms:
        assert hasattr(L, name), name
    assert sorted(sbp_b200.EXPORTED) == syms


def test_build_targets_sm100a_only():
    import importlib.util
    spec = importlib.util.spec_from_file_location("pkg_build", os.path.join(PKG, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    flags = " ".join(mod.NVCC_FLAGS)
    assert "arch=compute_100a,code=sm_100a" in flags
    assert os.path.exists(mod.LIB)


def test_no_cpu_fallback_without_device():
    import sbp_b200
    if sbp_b200.device_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(sbp_b200.SbpError) as e:
        sbp_b200.Graph(4, np.array([0, 1], np.int32), np.array([1, 2], np.int32))
    assert e.value.code == 2


def test_generator_is_deterministic_and_in_range():
    import dcsbm
    a = dcsbm.generate(V=500, K=7, alpha=1.0, gamma=2.5, kmin=10, kmax=100, w=0.6, seed=3)
    b = dcsbm.generate(V=500, K=7, alpha=1.0, gamma=2.5, kmin=10, kmax=100, w=0.6, seed=3)
    for x, y in zip(a[1:], b[1:]):
        assert np.array_equal(x, y)
    V, s, d, truth = a
    outdeg = np.bincount(s, minlength=V)
    assert outdeg.min() >= 10 and outdeg.max() <= 100
    assert s.max() < V and d.max() < V and truth.max() == 6
    assert len(np.unique(truth)) == 7
    frac_within = np.mean(truth[s] == truth[d])
    assert 0.55 < frac_within < 0.8


def test_batched_configs():
    import dcsbm
    sizes = [dcsbm.batched_config(g)["V"] for g in range(64)]
    assert min(sizes) >= 1000 and max(sizes) <= 50000
    c = dcsbm.batched_config(0)
    assert c["K"] == round(1.2 * c["V"] ** 0.35)


def test_engine_options_are_checked_on_the_host():
    """sbp_set_option validates names and ranges without a device; every option documented in
    the header is accepted at its default."""
    import sbp_b200 as S
    defaults = {"dense_max_blocks": 131072, "dense_max_memory_pct": 60, "hashed_row_factor": 4, "graph_sweeps": 1,
                "group_kernel": 1, "batched_wait_limit": 1 << 22, "batched_stall_graph": -1,
                "batched_overlap": 64, "batched_threads": 8}
    header = open(os.path.join(ROOT, "include", "sbp_b200.h")).read()
    for name, value in defaults.items():
        assert f'"{name}"' in header, name
        S.set_option(name, value)
    for name, bad in (("batched_threads", 0), ("batched_threads", 65), ("batched_overlap", -1),
                      ("group_kernel", 3), ("dense_max_memory_pct", 91), ("no_such_option", 1)):
        with pytest.raises(S.SbpError) as e:
            S.set_option(name, bad)
        assert e.value.code == 1
        assert name in S.last_error() or "option" in S.last_error()


def test_release_cached_memory_needs_no_device():
    import sbp_b200 as S
    S.release_cached_memory()   # nothing cached: no CUDA call
