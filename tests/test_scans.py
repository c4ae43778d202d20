"""
auto_slip.frame_differences and auto_slip.text_mask (python/slipcam/auto_slip.py:56-94): the oracle
restatement against the reference functions' own outputs (tests/golden/scans.npz, made by
make_scans.py), and the b200 scans (csrc/scans.cuh) against both.
"""

import os

import numpy as np
import pytest

from oracle import oracle


def golden():
    return dict(np.load(os.path.join(os.path.dirname(__file__), 'golden', 'scans.npz')))


def test_oracle_matches_reference_functions():
    g = golden()
    assert np.array_equal(oracle.frame_differences(g['frames']), g['diff'])
    assert np.array_equal(oracle.text_mask(g['frames'], 4, nframes=40, chunk=10), g['mask'])
    assert np.array_equal(oracle.text_mask(g['frames'], 6, nframes=30, chunk=6, edge_percentile=85, max_std=2.0,
                                           dilate=2), g['mask2'])


@pytest.mark.gpu
def test_b200_frame_differences():
    from slipcam_b200 import scans
    g = golden()
    d = scans.frame_differences(g['frames'], chunk=20)
    assert d.dtype == np.float32 and np.array_equal(d, g['diff'])


@pytest.mark.gpu
def test_b200_text_mask():
    from slipcam_b200 import scans
    g = golden()
    m = scans.text_mask(g['frames'], 4, nframes=40, chunk=10)
    assert m.dtype == bool and np.array_equal(m, g['mask'])
    m2 = scans.text_mask(g['frames'], 6, nframes=30, chunk=6, edge_percentile=85, max_std=2.0, dilate=2)
    assert np.array_equal(m2, g['mask2'])


@pytest.mark.gpu
def test_b200_text_mask_fills_a_large_box():
    """A ring as wide as the frame: the flood fill runs over many steps and fills it."""
    from slipcam_b200 import scans
    rng = np.random.default_rng(0)
    f = (128 + rng.integers(0, 12, (24, 300, 400))).astype(np.uint8)   # low-contrast flicker everywhere
    f[:, 20:24, 20:380] = f[:, 276:280, 20:380] = 250                  # a steady bright ring
    f[:, 20:280, 20:24] = f[:, 20:280, 376:380] = 250
    m = scans.text_mask(f, 0, nframes=20, chunk=10, dilate=1)
    assert m[150, 200] and m[22, 22] and not m[5, 5]
    assert np.array_equal(m, oracle.text_mask(f, 0, nframes=20, chunk=10, dilate=1))


@pytest.mark.gpu
@pytest.mark.parametrize('width,offset', [(167, 1), (168, 2), (150, 0), (33, 3)])
def test_frame_differences_any_alignment(width, offset):
    """The difference scan's 16-pixel, word and byte paths: frames at a base address `offset` bytes
    past an aligned one and of any width, through the C ABI, against the oracle."""
    import ctypes

    import torch
    from slipcam_b200 import _lib
    f = np.ascontiguousarray(golden()['frames'][:21, :, :width])
    n, h, w = f.shape
    buf = torch.zeros(n * h * w + 16, dtype=torch.uint8, device='cuda')
    buf[offset:offset + n * h * w] = torch.as_tensor(f.ravel()).cuda()
    out = torch.empty(n - 1, dtype=torch.float32, device='cuda')
    sums = torch.empty(n - 1, dtype=torch.int64, device='cuda')
    rc = _lib.lib().b200_frame_diff_device(buf.data_ptr() + offset, n, h, w, w, out.data_ptr(), sums.data_ptr(),
                                          torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.OK
    exact = np.array([np.abs(f[k + 1].astype(np.int64) - f[k].astype(np.int64)).sum() for k in range(n - 1)])
    assert np.array_equal(sums.cpu().numpy(), exact)
    np.testing.assert_array_equal(out.cpu().numpy(), oracle.frame_differences(f))
