import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and libp4a.so")


@pytest.fixture(scope="session")
def built():
    """Builds libp4a.so and the oracle library once per session if needed."""
    from particles4all_b200 import build as pbuild
    import oracle
    pbuild.build()
    oracle.build()
    return True
