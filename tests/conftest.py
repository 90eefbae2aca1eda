import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, 'three-avbd_b200'), os.path.join(ROOT, 'oracle'), os.path.join(ROOT, 'tests')):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a B200 (sm_100a) and the CUDA library')


@pytest.fixture(scope='session')
def cuda_lib():
    """The built CUDA library; GPU tests fail loudly if it is missing (no fallback)."""
    import avbd_b200
    return avbd_b200.load()
