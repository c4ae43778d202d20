"""Test configuration: the repository root and tests/golden on the path, the gpu marker."""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, 'tests', 'golden')):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a B200 (runs the CUDA library)')


@pytest.fixture(scope='session')
def oracle_mod():
    from oracle import oracle
    oracle.lib()
    return oracle
