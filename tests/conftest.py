import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "pacmap-rs_b200")
for p in (ROOT, PKG_DIR):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "reference_vectors.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def lib():
    """The product library (C ABI). Fails loudly if the CUDA build is missing."""
    import pacmap_b200

    return pacmap_b200


def gaussian_mixture(n, d, n_clusters=10, spread=5.0, sigma=1.0, seed=0):
    rng = np.random.default_rng(seed)
    centres = rng.normal(0.0, spread, size=(n_clusters, d)).astype(np.float32)
    lab = rng.integers(0, n_clusters, size=n)
    x = centres[lab] + rng.normal(0.0, sigma, size=(n, d)).astype(np.float32)
    return x.astype(np.float32), lab
