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
    assert np.array_equal(oracle.text_mask(g['frames'], 6, nframes=30, chunk=6, edge_percentile=85, max_std=2.0,
                                           dilate=0), g['mask0'])


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
    m0 = scans.text_mask(g['frames'], 6, nframes=30, chunk=6, edge_percentile=85, max_std=2.0, dilate=0)
    assert np.array_equal(m0, g['mask0'])


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


def test_text_mask_arguments_checked_before_any_launch():
    """Bad arguments come back as EINVAL from the C ABI without touching a device; the scratch size."""
    from slipcam_b200 import _lib
    lib = _lib.lib()
    assert lib.b200_text_mask_scratch_bytes(720, 1280) == _lib.PERCENTILE_SCRATCH + 2 * 720 * 40 * 4
    assert lib.b200_text_mask_scratch_bytes(0, 5) == 0
    assert lib.b200_percentile_f32_device(None, 10, 50.0, None, None, None) == _lib.EINVAL
    assert lib.b200_percentile_f32_device(1, 10, 100.5, 1, 1, None) == _lib.EINVAL
    assert lib.b200_percentile_f32_device(1, 10, float('nan'), 1, 1, None) == _lib.EINVAL
    assert lib.b200_percentile_f32_device(1, 0, 50.0, 1, 1, None) == _lib.EINVAL
    assert lib.b200_text_mask_device(1, 1, 4, 4, 90.0, 1.5, 4, 1, 1, 10, None) == _lib.EINVAL   # scratch too small
    assert lib.b200_text_mask_device(1, 1, 4, 40000, 90.0, 1.5, 4, 1, 1, 1 << 30, None) == _lib.EINVAL   # too wide


@pytest.mark.gpu
def test_b200_percentile_matches_numpy():
    """numpy.percentile of float32 data, bit for bit: negatives, ties, constant data, one value,
    q at 0 and 100, and a 720p edge map."""
    import torch
    from slipcam_b200 import scans
    rng = np.random.default_rng(11)
    cases = []
    for n in (1, 2, 3, 17, 1000, 4097, 100_003):
        x = (rng.standard_normal(n) * 50).astype(np.float32)
        cases += [x, np.round(x).astype(np.float32), np.abs(x), np.full(n, 2.5, np.float32)]
    g = golden()['frames'][0].astype(np.float32)
    cases.append(oracle._sobel_magnitude(g))
    cases.append((rng.random(720 * 1280) * 300).astype(np.float32))
    for x in cases:
        t = torch.as_tensor(x).cuda()
        for q in (0, 100, 90, 85, 50, 12.5, 99.9, 33.3):
            assert scans.percentile(t, q) == np.percentile(x, q), (x.size, q)


def _spiral(h, w, s=4):
    """Nested rectangular walls s pixels apart, each opened by a gap of s - 1 pixels, at the top
    left and the bottom right by turns: the background is one corridor that runs half way round
    every ring (still open after one dilation step, which narrows it to s - 3 pixels)."""
    m = np.zeros((h, w), bool)
    t, l, b, r, k = 2, 2, h - 3, w - 3, 0
    while b - t > s and r - l > s:
        m[t, l:r + 1] = m[b, l:r + 1] = m[t:b + 1, l] = m[t:b + 1, r] = True
        if k % 2 == 0:
            m[t + 1:t + s, l] = False
        else:
            m[b - s + 1:b, r] = False
        t, l, b, r, k = t + s, l + s, b - s, r - s, k + 1
    return m


def _mask_device(edge, sd, q, max_std, dilate):
    import torch
    from slipcam_b200 import _lib
    h, w = edge.shape
    lib = _lib.lib()
    e, s = torch.as_tensor(edge).cuda(), torch.as_tensor(sd).cuda()
    mask = torch.empty((h, w), dtype=torch.uint8, device='cuda')
    scratch = torch.empty(lib.b200_text_mask_scratch_bytes(h, w), dtype=torch.uint8, device='cuda')
    rc = lib.b200_text_mask_device(e.data_ptr(), s.data_ptr(), h, w, float(q), float(max_std), dilate, mask.data_ptr(),
                                   scratch.data_ptr(), scratch.numel(), torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.OK
    return mask.cpu().numpy().astype(bool)


@pytest.mark.gpu
@pytest.mark.parametrize('h,w', [(1, 1), (1, 70), (45, 1), (37, 70), (64, 96), (50, 129), (200, 333), (9, 2049),
                                 (6, 9000)])
def test_b200_mask_from_maps_random(h, w):
    """The threshold, dilation and hole filling on the device against the oracle (scipy labels):
    random seed masks of several densities, dilation 1, 4 and 11 (two launches of the tile
    dilation) and 0 (repeated until nothing changes: the whole frame once any pixel is set), rows of several words per lane in the horizontal sweep (2049 pixels) and wider than
    one of its segments (9000 pixels)."""
    rng = np.random.default_rng(h * 1000 + w)
    for dens in (0.02, 0.1, 0.3):
        edge = (rng.random((h, w)) * 100).astype(np.float32)
        sd = np.where(rng.random((h, w)) < 1 - dens, 5.0, 0.5).astype(np.float32)
        for q, dilate in ((90, 4), (50, 0), (99, 1), (0, 11)):
            got = _mask_device(edge, sd, q, 1.5, dilate)
            assert np.array_equal(got, oracle.mask_from_maps(edge, sd, q, 1.5, dilate)), (dens, q, dilate)


@pytest.mark.gpu
def test_b200_mask_fills_spirals_and_rings():
    """Shapes the sweeps need many rounds for: nested spirals (a corridor from the border that runs
    half way round every ring, up to about 4000 pixels long) and a ring inside a ring."""
    for h, w in ((41, 67), (120, 300), (257, 129), (20, 1300)):
        m = _spiral(h, w)
        edge, sd = np.where(m, 100.0, 1.0).astype(np.float32), np.zeros((h, w), np.float32)
        q = 100.0 * (1 - m.mean()) - 1e-3
        got = _mask_device(edge, sd, q, 1.5, 1)
        assert not got.all()   # the corridor stays open
        assert np.array_equal(got, oracle.mask_from_maps(edge, sd, q, 1.5, 1))
    m = np.zeros((90, 140), bool)
    m[5, 5:130] = m[80, 5:130] = True
    m[5:81, 5] = m[5:81, 129] = True
    m[20, 20:100] = m[60, 20:100] = True
    m[20:61, 20] = m[20:61, 99] = True
    m[20, 50] = False   # the inner ring opens into the outer ring's hole: both still enclosed
    edge, sd = np.where(m, 100.0, 1.0).astype(np.float32), np.zeros(m.shape, np.float32)
    got = _mask_device(edge, sd, 100.0 * (1 - m.mean()) - 1e-3, 1.5, 1)
    assert got[40, 60] and got[70, 60] and not got[2, 2]
    assert np.array_equal(got, oracle.mask_from_maps(edge, sd, 100.0 * (1 - m.mean()) - 1e-3, 1.5, 1))


@pytest.mark.gpu
@pytest.mark.parametrize('nchunks,chunk,width', [(15, 10, 1280), (1, 3, 77), (2, 5, 130), (4, 2, 128), (17, 2, 101),
                                                 (64, 1, 33)])
def test_b200_chunk_std_median(nchunks, chunk, width):
    """The temporal median of the chunks' deviations against the oracle: odd and even chunk counts,
    the register sort (up to 16 chunks) and the shared-memory one (17 and 64), widths that are not
    a multiple of 4 (the byte path)."""
    import torch
    from slipcam_b200 import _lib
    rng = np.random.default_rng(nchunks * 7 + width)
    h = 23
    f = rng.integers(0, 256, (nchunks * chunk, h, width), dtype=np.uint8)
    f[:, :5] = 128 + rng.integers(0, 2, (nchunks * chunk, 5, width), dtype=np.uint8)   # steady rows
    out = torch.empty((h, width), dtype=torch.float32, device='cuda')
    rc = _lib.lib().b200_chunk_std_median_device(torch.as_tensor(f).cuda().data_ptr(), nchunks, chunk, h, width, width,
                                                 out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.OK
    assert np.array_equal(out.cpu().numpy(), oracle.chunk_std_median(f, 0, nchunks * chunk, chunk))
