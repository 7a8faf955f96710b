import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "hybrid-stochastic-block-partitioning_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the engine through the C ABI")


@pytest.fixture(scope="session")
def S():
    """The engine binding; GPU tests fail loudly if the library or the device is missing."""
    import sbp_b200
    sbp_b200.load()
    if sbp_b200.device_count() < 1:
        raise RuntimeError("no CUDA device: GPU tests cannot run (the engine has no CPU fallback)")
    return sbp_b200


@pytest.fixture(scope="session")
def O():
    import sbp_oracle
    sbp_oracle.build()
    return sbp_oracle


def toy_fixture():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "toy_example.json")) as f:
        return json.load(f)


def random_graph(V, K, seed, kmin=4, kmax=40, w=0.7, alpha=3.0, gamma=2.5):
    import dcsbm
    return dcsbm.generate(V=V, K=K, alpha=alpha, gamma=gamma, kmin=kmin, kmax=kmax, w=w, seed=seed)


def random_assignment(V, B, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, B, V).astype(np.int32)
    a[:B] = rng.permutation(B)[:min(B, V)]
    return a


def random_records(n, seed):
    return np.random.default_rng(seed).integers(0, 2**32, size=(n, 4), dtype=np.uint64).astype(np.uint32)
