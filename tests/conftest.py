"""Shared test set-up: paths, the `gpu` marker, oracle and library fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "sinking-simulator_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path through the C ABI")


@pytest.fixture(scope="session")
def port():
    import oracle

    return oracle.Oracle("port")


@pytest.fixture(scope="session")
def ref():
    import oracle

    if not oracle.have_ref():
        pytest.skip("the compiled reference (oracle/_ref) is not built here")
    return oracle.Oracle("ref")


@pytest.fixture(scope="session")
def fem():
    """The product binding.  On a GPU test, a missing device is a failure, not a skip."""
    import femstep

    return femstep
