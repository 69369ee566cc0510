import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# The oracle's searches run one orientation chunk per OpenMP thread, each with
# about 1 GB of FP64 buffers at 4096^2: cap the threads before it loads.
os.environ.setdefault("OMP_NUM_THREADS", str(max(1, min(os.cpu_count() or 1, 16))))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built sm_100a library")
    config.addinivalue_line("markers", "slow: longer CPU test")


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(ROOT, "tests", "golden")
