import faulthandler
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


# A test that runs past BN_TEST_LIMIT_S seconds (default 300; the whole GPU
# suite takes about a minute) dumps every thread's stack to stderr and ends
# the run, so a stall shows where it happened instead of using up the
# caller's time limit.
_TEST_LIMIT_S = float(os.environ.get("BN_TEST_LIMIT_S", "300"))


@pytest.hookimpl(hookwrapper=True)
def pytest_runtest_protocol(item, nextitem):
    if _TEST_LIMIT_S > 0:
        faulthandler.dump_traceback_later(_TEST_LIMIT_S, exit=True, file=sys.__stderr__)
    try:
        yield
    finally:
        if _TEST_LIMIT_S > 0:
            faulthandler.cancel_dump_traceback_later()


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
