import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "sycl-optic-flow_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and liboflow.so")


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.orc_lib()
    return oracle


@pytest.fixture(scope="session")
def ref():
    import oracle
    if not oracle.ref_available():
        pytest.skip("reference TV-L1 (oracle/_ref) not built here")
    oracle.ref_lib()
    return oracle


@pytest.fixture(scope="session")
def of():
    """The GPU library: no fallback, a missing build or device is an error."""
    import oflow
    oflow.capi.lib()
    return oflow


@pytest.fixture(scope="session")
def ctx(of):
    c = of.Context(0)
    yield c
    c.close()
