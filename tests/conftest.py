"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu)")
    config.addinivalue_line("markers", "slow: long-running (still part of the default run)")


@pytest.fixture(scope="session")
def orc():
    import oracle
    if not os.path.exists(oracle.restated_path()):
        import subprocess
        subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "restated"])
    return oracle.restated()


@pytest.fixture(scope="session")
def gpu():
    import bluecrunch_b200 as bc
    bc.init(0)
    yield bc


def limbs(seed, n):
    import oracle
    return oracle.random_limbs(seed, n)


def exact(a, b, CL):
    """Exact product mod 2^(32 CL) with Python integers (small/medium sizes)."""
    import bluecrunch_b200 as bc
    return bc.from_int(bc.to_int(a) * bc.to_int(b) % (1 << (32 * CL)), CL)
