"""
The error paths, exercised without a GPU fault (the reference wraps every CUDA call and turns its
status into a "framecor: " runtime error, cxx/cuda.cu:28-40):

* a bounded device wait that nothing completes gives up and reports B200_ETIMEOUT, and the context
  stays usable (b200_wait_selftest: no MMA or copy is in flight while it waits);
* an allocation failure, injected on the host, surfaces as RuntimeError with a "framecor: " message
  from the constructor and from the first host-path call, and the next attempt succeeds;
* device-path callers read the status word with check(); a clean run reports nothing.
"""

import numpy as np
import pytest

from slipcam_b200 import _lib, framecor, synth

torch = pytest.importorskip('torch')


def test_entry_points_exported():
    for name in ('b200_status', 'b200_inject_alloc_failure', 'b200_wait_selftest'):
        assert hasattr(_lib.lib(), name)
    assert _lib.lib().b200_inject_alloc_failure(-1) == _lib.EINVAL
    assert _lib.lib().b200_inject_alloc_failure(0) == _lib.OK


@pytest.mark.gpu
def test_bounded_wait_gives_up_and_context_survives():
    stream = torch.cuda.current_stream().cuda_stream
    assert _lib.lib().b200_wait_selftest(1000, 1.0, stream) == _lib.ETIMEOUT
    x = torch.arange(1024, device='cuda', dtype=torch.float32)   # the context still works
    assert float(x.sum()) == 1023 * 1024 / 2
    frames = synth.video(240, 320, 2, np.array([[0.0, 0.0], [1.2, -0.7]]), np.zeros(2), seed=4)
    down, across = framecor.window_grid(240, 320, 32, 8, 32)
    cor = framecor.Correlator(240, 320, down, across, window=32, search=8, backend='b200')
    cor.set_reference(frames[0])
    r = cor.correlate(frames[1:])
    assert np.isfinite(r['offsets']).mean() > 0.9


@pytest.mark.gpu
@pytest.mark.parametrize('nth', [1, 2, 5])
def test_injected_allocation_failure_in_constructor(nth):
    down, across = framecor.window_grid(240, 320, 64, 16, 32)
    _lib.lib().b200_inject_alloc_failure(nth)
    try:
        with pytest.raises(RuntimeError, match=r'^framecor: .*out of memory \(injected\)'):
            framecor.Correlator(240, 320, down, across, window=64, search=16, backend='b200')
    finally:
        _lib.lib().b200_inject_alloc_failure(0)
    framecor.Correlator(240, 320, down, across, window=64, search=16, backend='b200')   # then it works


@pytest.mark.gpu
def test_injected_allocation_failure_in_first_call():
    frames = synth.video(240, 320, 2, np.array([[0.0, 0.0], [0.4, 0.3]]), np.zeros(2), seed=5)
    down, across = framecor.window_grid(240, 320, 32, 8, 32)
    cor = framecor.Correlator(240, 320, down, across, window=32, search=8, backend='b200')
    cor.set_reference(frames[0])
    _lib.lib().b200_inject_alloc_failure(1)   # the host path's slots are allocated by its first call
    try:
        with pytest.raises(RuntimeError, match=r'^framecor: cudaMalloc: out of memory \(injected\)'):
            cor.correlate(frames[1:])
    finally:
        _lib.lib().b200_inject_alloc_failure(0)
    r = cor.correlate(frames[1:])   # nothing was left half-built
    assert np.isfinite(r['offsets']).mean() > 0.9


@pytest.mark.gpu
def test_device_path_status_clean():
    c_frames, motion, step, gross = synth.hd(n=3, count=3, device='cuda')
    down, across = framecor.window_grid(720, 1280, 64, 48, 16)
    cor = framecor.Correlator(720, 1280, down, across, window=64, search=48, backend='b200')   # tensor-core form
    cor.set_reference(c_frames[0])
    cor.correlate(c_frames[1:], gross=torch.as_tensor(gross[1:]).cuda())
    cor.check()   # nothing gave up
