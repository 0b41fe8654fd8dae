import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def pkg():
    """The product package (directory name contains a hyphen)."""
    return importlib.import_module("fyzzxyzzy-sdk_b200")


@pytest.fixture(scope="session")
def scenes():
    return importlib.import_module("fyzzxyzzy-sdk_b200.scenes")


@pytest.fixture(scope="session")
def oracle():
    import oraclescene
    oraclescene.lib()
    return oraclescene


@pytest.fixture(scope="session")
def ref():
    import refscene
    if not refscene.available():
        pytest.skip("reference NativeCpu harness not built (oracle/_ref)")
    return refscene
