import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, 'tests', 'golden')
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, 'oracle'))


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200)')


@pytest.fixture(scope='session')
def known():
    with open(os.path.join(GOLDEN, 'known_answers.json')) as f:
        return {k: v['value'] for k, v in json.load(f).items()}


@pytest.fixture(scope='session')
def refvec():
    return np.load(os.path.join(GOLDEN, 'reference_vectors.npz'))


@pytest.fixture(scope='session')
def oracle():
    import oracle as O
    return O


@pytest.fixture(scope='session')
def basis_library():
    with open(os.path.join(ROOT, 'napmo_b200', 'data', 'basis.json')) as f:
        return json.load(f)


@pytest.fixture(scope='session')
def elements():
    with open(os.path.join(ROOT, 'napmo_b200', 'data', 'elements.json')) as f:
        return json.load(f)


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
