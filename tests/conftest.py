import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device")


def load_fixture(name):
    """A golden fixture as the dict form the oracle and the force take."""
    d = dict(np.load(os.path.join(GOLDEN, name)))
    for k in ("coulomb_scaling", "cellsize", "ron", "rc_lj", "rc_coul", "rc_alg",
              "golden_elj", "golden_ecoul"):
        if k in d:
            d[k] = float(d[k])
    d["n"] = int(d["type"].size)
    return d


@pytest.fixture(scope="session")
def water423():
    return load_fixture("water423.npz")


@pytest.fixture(scope="session")
def water648():
    return load_fixture("water648_ref.npz")


@pytest.fixture(scope="session")
def modified648():
    return load_fixture("modified_ref.npz")
