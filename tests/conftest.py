import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "parallel-randomized-cholesky_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs through the C-ABI library")
    config.addinivalue_line("markers", "slow: takes minutes (benchmark-size inputs)")


@pytest.fixture(scope="session")
def gpu_ctx_factory():
    import rchol_b200 as R

    made = []

    def make(**kw):
        c = R.Context(**kw)
        made.append(c)
        return c

    yield make
    for c in made:
        c.close()
