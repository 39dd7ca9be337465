import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden_small():
    return dict(np.load(os.path.join(GOLDEN, "small_pmis.npz")))


@pytest.fixture(scope="session")
def golden_edge():
    return dict(np.load(os.path.join(GOLDEN, "edge_cases.npz")))


@pytest.fixture(scope="session")
def golden_digests():
    import json
    return json.load(open(os.path.join(GOLDEN, "digests.json")))


@pytest.fixture(scope="session")
def oracle():
    import ref
    if not ref.have_oracle():
        import subprocess
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle_amg.so"],
                       check=True, capture_output=True)
    return ref
