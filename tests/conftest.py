import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (runs the sm_100a kernels through the C ABI)')


@pytest.fixture(scope='session')
def oracle():
    from oracle import oracle as O
    O.load()
    return O


@pytest.fixture(scope='session')
def pbso4():
    from powder6_b200.workloads import wyckoff_problem
    return wyckoff_problem(seed=1)
