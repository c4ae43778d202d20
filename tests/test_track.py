"""
The streaming driver (slipcam_b200.track): the reference driver's arguments and .npz keys
(python/slipcam/track_offsets.py:35-60), outputs identical to one Correlator.correlate over the
same frames, chunk after chunk from a memory-mapped video.
"""

import numpy as np
import pytest

from slipcam_b200 import framecor, synth, track

KEYS = {'index', 'ref', 'masked', 'yc', 'xc', 'window', 'skip', 'search', 'engine', 'offsets', 'snr', 'cov', 'peak'}


def test_boxes_mask_matches_brute_force():
    y0, x0 = framecor.window_grid(360, 640, 32, 16, 16)
    boxes = [(100, 20, 300, 60), (500, 300, 640, 360)]
    m = track.boxes_mask(y0, x0, 32, boxes)
    for i, y in enumerate(y0):
        for j, x in enumerate(x0):
            hit = any(x < bx1 and x + 32 > bx0 and y < by1 and y + 32 > by0 for bx0, by0, bx1, by1 in boxes)
            assert m[i, j] == hit


def test_cpu_refused():
    with pytest.raises(ValueError, match='no CPU path'):
        track.track(np.zeros((2, 64, 64), np.uint8), 0, [1], window=16, skip=16, search=4, cpu=True)


@pytest.mark.gpu
def test_track_cli_matches_correlate(tmp_path):
    torch = pytest.importorskip('torch')
    frames, motion, _ = synth.small(n=21)
    path = tmp_path / 'frames.npy'
    np.save(path, frames)
    out = tmp_path / 'offsets.npz'
    track.main([str(path), '--ref', '0', '--first', '1', '--window', '32', '--search', '16', '--skip', '16',
                '--chunk', '8', '--mask', '100', '20', '300', '60', '--out', str(out)])
    r = dict(np.load(out))
    assert set(r) == KEYS
    y0, x0 = framecor.window_grid(360, 640, 32, 16, 16)
    cor = framecor.Correlator(360, 640, y0, x0, window=32, search=16, backend='b200')
    cor.set_reference(frames[0])
    want = cor.correlate(frames[1:])
    for key in ('offsets', 'snr', 'cov', 'peak'):
        assert np.array_equal(r[key], want[key], equal_nan=True), key
    assert np.array_equal(r['index'], np.arange(1, 21)) and r['masked'].sum() > 0
    assert np.allclose(r['yc'], y0 + 16) and str(r['engine']) == 'framecor'
    err = np.abs(r['offsets'] - motion[1:, None, None, :])
    assert np.nanmedian(err) < 0.1


@pytest.mark.gpu
def test_track_gathers_scattered_frames():
    frames, _, _ = synth.small(n=12)
    y0, x0 = framecor.window_grid(360, 640, 32, 16, 16)
    idx = np.array([11, 3, 5, 7, 2])
    r = track.track(frames, 0, idx, window=32, skip=16, search=16, chunk=2)
    cor = framecor.Correlator(360, 640, y0, x0, window=32, search=16, backend='b200')
    cor.set_reference(frames[0])
    want = cor.correlate(frames[idx])
    assert np.array_equal(r['offsets'], want['offsets'], equal_nan=True)
