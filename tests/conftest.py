import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "B32p1e4.npz"))


@pytest.fixture(scope="session")
def golden_ic_positions():
    import numpy as np
    # bfps/DNS.py:711-733 with --particle-rand-seed 2
    np.random.seed(2)
    return np.random.random((10000, 3)) * 2 * np.pi
