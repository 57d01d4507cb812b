"""Shared fixtures.  `-m gpu` tests need a CUDA device and the built native library;
everything else runs on the CPU (oracle, host logic, C-ABI symbol checks)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200) and libnipet_b200.so')
    config.addinivalue_line('markers', 'slow: long-running CPU test')


@pytest.fixture(scope='session')
def params():
    from nipet_b200 import geometry
    return geometry.get_mmrparams()


@pytest.fixture(scope='session')
def oracle(params):
    from oracle import oracle as O
    return O.Oracle(params)


@pytest.fixture(scope='session')
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch.device('cuda', 0)


def phantom(seed=0, kind='brain'):
    from nipet_b200 import phantoms
    return phantoms.brain_phantom(seed=seed) if kind == 'brain' else phantoms.random_ellipsoids(seed=seed)
