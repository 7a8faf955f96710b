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
