"""Shared test set-up: import paths, the gpu marker, golden-vector loading."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, 'wind-tunnel_b200')
ORACLE = os.path.join(ROOT, 'oracle')
GOLDEN = os.path.join(ROOT, 'tests', 'golden')
for p in (ROOT, PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (a B200 for the timing-sensitive ones)')


def golden(name):
    with np.load(os.path.join(GOLDEN, name)) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope='session')
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


def has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
