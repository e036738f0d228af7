import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a) device")
    config.addinivalue_line("markers", "slow: large workloads (seconds of GPU time)")


@pytest.fixture(scope="session")
def gsr_ctx_factory():
    from rustscan_b200 import Context

    made = []

    def make(**kw):
        c = Context(**kw)
        made.append(c)
        return c

    yield make
    for c in made:
        c.close()
