import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# the oracle's OpenMP reductions sum in an order fixed by the thread count: one count on every
# host keeps the checker's rounding, and so the iteration counts of the sensitive BiCGStab
# variants, the same everywhere (set before the OpenMP runtime starts)
os.environ.setdefault("OMP_NUM_THREADS", "8")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a library")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O
