import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "cubism-jr-gpu-mpcf_b200")
for p in (PKG, os.path.join(REPO, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def mpcf():
    import mpcf as m
    return m


def cloud_state(dims, nb=2, seed=11, p_liquid=100.0, dtype=np.float32):
    """Host-generated bubble-cloud state (7 flat arrays) for a domain."""
    import mpcf as m
    params, bub = m.configs.small_cloud(dims, nb=nb, seed=seed, p_liquid=p_liquid)
    return m.ic_cloud_host(dims, params, bub, dtype=dtype)
