"""
The pinned staging of host frames (slipcam_b200/_stage.py): the split copies on the CPU, and the
round trip through the device on the GPU with sources that are not one contiguous block.
"""

import numpy as np
import pytest

from slipcam_b200 import _stage


@pytest.mark.parametrize('shape', [(1, 1, 1), (3, 5, 7), (40, 720, 130), (9, 1000, 1000)])
def test_parallel_copy_contiguous_and_strided(shape):
    rng = np.random.default_rng(sum(shape))
    src = rng.integers(0, 256, shape, dtype=np.uint8)
    for view in (src, src[::-1], src[:, ::2], src[::2, :, 1:]):
        dst = np.empty(view.shape, np.uint8)
        _stage.parallel_copy(dst, view)
        assert np.array_equal(dst, view)


def test_host_copy_any_alignment_and_size():
    """b200_host_copy (streaming stores past the destination's first 16-byte boundary, plain copies at
    the ends) moves every byte, at every source and destination offset; no GPU is touched."""
    from slipcam_b200 import _lib
    lib = _lib.lib()
    rng = np.random.default_rng(8)
    src = rng.integers(0, 256, 1 << 16, dtype=np.uint8)
    for so, do, n in [(0, 0, 0), (0, 0, 1), (3, 5, 17), (1, 15, 64), (7, 0, 65), (0, 9, 4095), (13, 2, 40000)]:
        dst = np.zeros(n + 64, np.uint8)
        assert lib.b200_host_copy(dst.ctypes.data + do, src.ctypes.data + so, n) == _lib.OK
        assert np.array_equal(dst[do:do + n], src[so:so + n])
        assert not dst[:do].any() and not dst[do + n:].any()
    assert lib.b200_host_copy(None, src.ctypes.data, 5) == _lib.EINVAL


def test_parallel_copy_from_a_memory_map(tmp_path):
    rng = np.random.default_rng(3)
    a = rng.integers(0, 256, (12, 300, 401), dtype=np.uint8)
    path = tmp_path / 'frames.u8'
    a.tofile(path)
    mm = np.memmap(path, dtype=np.uint8, mode='r', shape=a.shape)
    dst = np.empty((5, 300, 401), np.uint8)
    _stage.parallel_copy(dst, mm[4:9])
    assert np.array_equal(dst, a[4:9])


@pytest.mark.gpu
def test_upload_and_download_round_trip():
    """Chunks of a host array through three pinned buffers to the device and back through two,
    including a short last chunk and a reversed (negative-stride) source."""
    import torch
    rng = np.random.default_rng(7)
    a = rng.integers(0, 256, (23, 97, 131), dtype=np.uint8)
    dev = torch.empty(a.shape, dtype=torch.uint8, device='cuda')
    up = _stage.Uploader(a.shape[1:], 5, dev.device)
    stream = torch.cuda.current_stream()
    for k in range(0, len(a), 5):
        stream.wait_event(up.put(a[::-1][k:k + 5], dev[k:k + 5]))
    out = np.zeros_like(a)
    down = _stage.Downloader(a.shape[1:], 5, dev.device)
    for k in range(0, len(a), 5):
        down.get(dev[k:k + 5], out[k:k + 5], after=stream.record_event())
    down.flush()
    assert np.array_equal(out, a[::-1])
