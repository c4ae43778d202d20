"""
auto_slip.periodicity (python/slipcam/auto_slip.py:105-129): the oracle restatement against the
reference function's own outputs (tests/golden/periodicity.npz, made by make_periodicity.py), and the
b200 version (FP32 surfaces, the peak search on the GPU) against both.
"""

import numpy as np
import pytest

from oracle import oracle

GOLDEN = None


def golden():
    global GOLDEN
    if GOLDEN is None:
        import os
        GOLDEN = dict(np.load(os.path.join(os.path.dirname(__file__), 'golden', 'periodicity.npz')))
    return GOLDEN


def case(k):
    g = golden()
    w, s, e = (int(x) for x in g[f'geom{k}'])
    return g[f'ref{k}'], g[f'y0{k}'], g[f'x0{k}'], w, s, e, g[f'out{k}']


@pytest.mark.parametrize('k', [0, 1])
def test_oracle_matches_reference_function(k):
    ref, y0, x0, w, s, e, out = case(k)
    assert np.abs(oracle.periodicity(ref, y0, x0, w, s, e) - out).max() < 1e-8


@pytest.mark.gpu
@pytest.mark.parametrize('k', [0, 1])
def test_b200_periodicity(k):
    from slipcam_b200 import framecor
    ref, y0, x0, w, s, e, out = case(k)
    got = framecor.periodicity(ref, y0, x0, w, s, e)
    assert got.shape == out.shape and got.dtype == np.float64
    assert np.all(got[out == 1.0] == 1.0)                  # the flat windows (periodic ones come near 1)
    assert np.abs(got - out).max() < 1e-4, np.abs(got - out).max()
