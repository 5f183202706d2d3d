import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "blastp-cuda_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def matrix():
    """The reference's BLOSUM62 (NCBIstdaa 28x28) from the committed fixture."""
    path = os.path.join(ROOT, "tests", "golden", "blosum62_ncbistdaa.txt")
    return np.loadtxt(path, dtype=np.int64).astype(np.int8)


@pytest.fixture(scope="session")
def engine():
    from blastp_b200 import Engine
    e = Engine(0)
    yield e
    e.close()
