"""Shared fixtures.  Tests marked `gpu` need a CUDA device and the built
library; everything else runs on CPU (the oracle, host logic, the C ABI's
symbol table)."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built sm_100a library")


@pytest.fixture(scope="session")
def built():
    """Build (if stale) the product library and the oracle."""
    from tdfs_b200 import build as b
    b.build()
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    import tdfs_b200
    return tdfs_b200


@pytest.fixture(scope="session")
def T(built):
    return built


@pytest.fixture(scope="session")
def po():
    from oracle import pyoracle
    pyoracle.build()
    return pyoracle
