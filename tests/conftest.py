import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libb3g.so")
    config.addinivalue_line("markers", "slow: longer CPU checks")


@pytest.fixture(scope="session")
def port():
    import oracle

    oracle.build(port=True, ref=False)
    return oracle


@pytest.fixture(scope="session")
def b3g():
    import bounce_b200
    from bounce_b200 import build

    build.build()
    bounce_b200.lib()
    return bounce_b200
