import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200) and the built library')


@pytest.fixture(scope='session')
def golden3d():
    import numpy as np
    return np.load(os.path.join(ROOT, 'tests', 'golden', 'generic_euler_3d.npz'))


@pytest.fixture(scope='session')
def golden2d():
    import numpy as np
    return np.load(os.path.join(ROOT, 'tests', 'golden', 'generic_euler_2d.npz'))
