"""
The no-allocation entry point, b200_correlate_device_noalloc, for callers that cannot allocate
device memory while they correlate (a capture loop that must not stall on cudaMalloc, a host that
owns all device memory). It keeps its per-frame tables in a static device array instead of the
handle's buffers; it always runs the FP32 form, and its outputs must match b200_correlate_device's
with that form, call after call, at the FFT sizes 160, 192 and 256 (the big transform's clusters).

This file is collected last on purpose (pytest -x stops at it only after every other test ran).
"""

import ctypes

import numpy as np
import pytest

from slipcam_b200 import _lib, framecor, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')

TOL = 1e-6   # the same kernels on the same inputs: the results agree to the last bit in practice


def run(entry, cor, frames, gross):
    n, ny, nx = frames.shape[0], *cor.shape
    out = [torch.empty((n, ny, nx, 2), dtype=torch.float32, device='cuda'),
           torch.empty((n, ny, nx), dtype=torch.float32, device='cuda'),
           torch.empty((n, ny, nx), dtype=torch.float32, device='cuda'),
           torch.empty((n, ny, nx, 3), dtype=torch.float32, device='cuda')]
    stream = torch.cuda.current_stream().cuda_stream
    rc = getattr(_lib.lib(), entry)(cor._h, frames.data_ptr(), n, frames.shape[2], gross.data_ptr(),
                                    _lib.GROSS_FRAME, *[o.data_ptr() for o in out], stream)
    _lib.raise_for(rc, cor._h)
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in out]


def same(a, b):
    for x, y in zip(a, b):
        assert np.array_equal(np.isnan(x), np.isnan(y))
        ok = np.isfinite(x)
        assert np.abs(x[ok] - y[ok]).max(initial=0.0) <= TOL


@pytest.mark.parametrize('window, search, skip', [(64, 48, 16), (64, 64, 48), (128, 64, 64)])
def test_noalloc_matches_device_entry_point(window, search, skip):
    """Two calls in a row on different frames: each matches the allocating entry point."""
    frames, motion, step, gross = synth.hd(n=12, count=12, device='cuda')
    g = torch.as_tensor(gross).cuda()
    down, across = framecor.window_grid(720, 1280, window, search, skip)
    cor = framecor.Correlator(720, 1280, down, across, window=window, search=search, backend='b200')
    cor.set_form('fft32')   # the form the no-allocation entry point runs
    cor.set_reference(frames[0])
    for first, last in ((1, 6), (6, 12)):
        f, gg = frames[first:last].contiguous(), g[first:last].contiguous()
        cor.set_form('fft32')
        expect = run('b200_correlate_device', cor, f, gg)
        got = run('b200_correlate_device_noalloc', cor, f, gg)
        same(expect, got)
        assert np.isfinite(got[0]).mean() > 0.9
        cor.set_form('auto')   # the handle's form does not reach the no-allocation entry point
        same(expect, run('b200_correlate_device_noalloc', cor, f, gg))


def test_noalloc_rejects_frames_too_large():
    """Tables beyond the 32 MiB static array: a clear error, nothing run."""
    h, w = 1440, 2560
    down, across = framecor.window_grid(h, w, 32, 8, 8)   # many windows: one frame per launch group
    cor = framecor.Correlator(h, w, down, across, window=32, search=8, backend='b200')
    cor.set_reference(np.full((h, w), 9, np.uint8))
    frames = torch.zeros((1, h, w), dtype=torch.uint8, device='cuda')
    gross = torch.zeros((1, 2), dtype=torch.int32, device='cuda')
    with pytest.raises(ValueError, match='too large for the no-allocation entry point'):
        run('b200_correlate_device_noalloc', cor, frames, gross)


def test_noalloc_is_declared_and_exported():
    assert hasattr(_lib.lib(), 'b200_correlate_device_noalloc')
    assert isinstance(_lib.lib().b200_correlate_device_noalloc, ctypes._CFuncPtr)
