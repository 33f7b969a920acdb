# -*- coding: utf-8 -*-
import os
import sys
import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, 'tests', 'golden')


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device (B200, sm_100a) and the built "
                   "extension; the parity tests proper")


@pytest.fixture(scope='session')
def golden_transforms():
    return dict(np.load(os.path.join(GOLDEN, 'transforms.npz')))


@pytest.fixture(scope='session')
def golden_params():
    return dict(np.load(os.path.join(GOLDEN, 'host_params.npz')))


@pytest.fixture(scope='session')
def golden_digests():
    return dict(np.load(os.path.join(GOLDEN, 'digests.npz')))
