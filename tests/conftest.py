"""Test configuration: package paths and the ``gpu`` marker.

Tests marked ``gpu`` need a CUDA device and the built libnhflood.so; the
rest run on the CPU (oracle, host logic, the C ABI's exported symbols).
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / 'nh-flood-2d_b200', ROOT / 'oracle', ROOT / 'tests'):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))
os.environ.setdefault('OMP_NUM_THREADS', str(min(8, os.cpu_count() or 1)))


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200) and libnhflood.so')
    config.addinivalue_line('markers', 'slow: longer CPU runs')


@pytest.fixture(scope='session')
def cuda_available():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return True
