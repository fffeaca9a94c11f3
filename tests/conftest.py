import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle_built():
    from oracle import bind
    bind.build_oracle()
    return True


@pytest.fixture(scope="session")
def reference_available():
    from oracle.bind import Reference
    if not Reference.available():
        pytest.skip("reference build (oracle/_ref) not present")
    return True
