import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) and the built libiqcp_gpu.so")
    config.addinivalue_line("markers", "slow: larger oracle runs (minutes)")


def golden(name):
    import json
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.lib()
    return oracle


def random_density(nbf, seed=0, scale=0.2):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(nbf, nbf)) * scale
    return A + A.T
