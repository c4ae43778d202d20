"""
The exact tensor-core form (set_form('int8'), B200_FORM_I8): the correlation summed directly on the
tensor cores in integers, then normalized.

* its tensor-core path against a host GEMM, exactly (b200_tc_i8_selftest): the A operand in TMEM or
  shared memory, the search window in shared memory as the kernel holds it, started at row i;
* every golden case against the FP64 direct-correlation oracle with gates tighter than the FP32
  form's: offsets within 1e-4 px, SNR within 1e-5 relative, peak within 1e-6, integer peaks
  identical except verified near-ties;
* the normalized surfaces against the oracle's FP64 surfaces within 2e-6 (the numerator is exact;
  only the FP32 variance denominator and the final roundings remain);
* the reference CPU backend's outputs (tests/golden) with the reference test's CPU/CUDA agreement
  bounds;
* geometries across the kernel's range: odd and tiny windows, searches above 63 px (two lane tiles
  of shifts), window 128 with search 64 (L = 256), several launches of frames (frames in rows off
  16-byte boundaries, which the Python device path would make contiguous, go through the C entry
  point with a pitch in test_parity.py).
"""

import numpy as np
import pytest

import cases
from oracle import oracle
from slipcam_b200 import _lib, framecor, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')

NEAR_TIE = 1e-5


@pytest.mark.parametrize('a_smem', [1, 0])
@pytest.mark.parametrize('n, k, rows, i', [(16, 32, 16, 0), (112, 160, 175, 63), (48, 64, 79, 31), (144, 256, 271, 127),
                                            (256, 32, 300, 44), (32, 96, 40, 7)])
def test_mma_i8(n, k, rows, i, a_smem):
    rng = np.random.default_rng(n * 1000 + k + i)
    a = rng.integers(0, 256, (128, k), dtype=np.uint8)
    x = rng.integers(0, 256, (rows, k), dtype=np.uint8)
    da, dx = torch.as_tensor(a).cuda(), torch.as_tensor(x).cuda()   # held until the call returns
    d = torch.empty((128, n), dtype=torch.int32, device='cuda')
    rc = _lib.lib().b200_tc_i8_selftest(da.data_ptr(), dx.data_ptr(), d.data_ptr(), n, k, rows, i, a_smem,
                                        torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.OK
    ref = a.astype(np.int64) @ x[i:i + n].astype(np.int64).T
    assert np.array_equal(d.cpu().numpy().astype(np.int64), ref)


def correlator(c, form='int8'):
    cor = framecor.Correlator(c['height'], c['width'], c['down'], c['across'], window=c['window'],
                              search=c['search'], stat_size=c['stat_size'], backend='b200')
    cor.set_form(form)
    cor.set_reference(c['reference'])
    return cor


def near_ties(c, mism, b, sl):
    """Every mismatched integer peak is a near-tie on the FP64 surface: the value at b's peak is
    within NEAR_TIE of the maximum."""
    if not mism.any():
        return True
    R = c['search']
    g = oracle.expand_gross(c['gross'], len(c['frames']), len(c['down']), len(c['across']))
    down, across = c['down'][sl[1]], c['across'][sl[2]]
    for f, y, x in np.argwhere(mism):
        gg = None if g is None else g[sl][f:f + 1, y:y + 1, x:x + 1]
        s = oracle.correlate(c['height'], c['width'], down[y:y + 1], across[x:x + 1], c['reference'],
                             c['frames'][f:f + 1], gg, window=c['window'], search=R, stat_size=c['stat_size'],
                             mode='f64', surfaces=True)['surface'][0, 0, 0]
        gy, gx = (0, 0) if gg is None else gg[0, 0, 0]
        u = int(np.rint(b['offsets'][f, y, x, 0] - gy + R))
        v = int(np.rint(b['offsets'][f, y, x, 1] - gx + R))
        if s.max() - s[u, v] > NEAR_TIE:
            return False
    return True


@pytest.mark.parametrize('name', list(cases.NAMES))
def test_fp64_oracle(name):
    c = cases.case(name)
    r = correlator(c).correlate(c['frames'], gross=c['gross'])
    a, b = cases.SUBGRID.get(name, (1, 1))
    sl = (slice(None), slice(None, None, a), slice(None, None, b))
    down, across, gross = c['down'][sl[1]], c['across'][sl[2]], c['gross']
    o = oracle.correlate(c['height'], c['width'], down, across, c['reference'], c['frames'],
                         gross if gross is None or gross.ndim == 2 else gross[sl], window=c['window'],
                         search=c['search'], stat_size=c['stat_size'], mode='f64')
    b = {k: v[sl] for k, v in r.items()}
    assert np.array_equal(np.isnan(o['offsets']), np.isnan(b['offsets']))
    valid = np.isfinite(o['offsets'][..., 0])
    assert np.all(b['snr'][~valid] == 0) and np.all(b['peak'][~valid] == 0)
    assert np.all(b['cov'][~valid] == np.array([99, 99, 0], np.float32))
    d = np.abs(o['offsets64'] - b['offsets']).max(-1)
    mism = valid & (d > 0.1)
    assert near_ties(c, mism, b, sl)
    ok = valid & ~mism
    assert d[ok].max() < 1e-4, d[ok].max()
    assert np.abs(b['snr'][ok] / o['snr'][ok] - 1).max() < 1e-5
    assert np.abs(b['peak'][ok] - o['peak'][ok]).max() < 1e-6


@pytest.mark.parametrize('name', list(cases.NAMES))
def test_golden(name):
    """Against the reference CPU backend's own outputs (FFT in FP32): the reference test's bounds."""
    c = cases.case(name)
    g = dict(np.load(f'{cases.__file__.rsplit("/", 1)[0]}/{name}.npz'))
    r = correlator(c).correlate(c['frames'], gross=c['gross'])
    a, b = g['offsets'], r['offsets']
    assert np.array_equal(np.isnan(a), np.isnan(b))
    valid = np.isfinite(a[..., 0])
    d = np.abs(a - b).max(-1)
    mism = valid & (d > 0.1)
    assert near_ties(c, mism, r, (slice(None),) * 3)   # the reference's own rounding decides only ties
    ok = valid & ~mism
    assert d[ok].max() < 1e-3
    assert np.abs(g['peak'][ok] - r['peak'][ok]).max() < 1e-4
    assert np.abs(r['snr'][ok] / g['snr'][ok] - 1).max() < 1e-2


def surfaces_vs_oracle(h, w, window, search, frames, gross=None, skip=24, limit=(3, 4), pitch_offset=0):
    down, across = framecor.window_grid(h, w, window, search, skip)
    down, across = down[:limit[0]], across[:limit[1]]
    cor = framecor.Correlator(h, w, down, across, window=window, search=search, backend='b200')
    cor.set_form('int8')
    cor.set_reference(frames[0])
    t = torch.as_tensor(frames[1:]).cuda()
    if pitch_offset:   # a strided view (correlate copies it contiguous; the pitch path is in test_parity.py)
        big = torch.zeros((t.shape[0], h, w + pitch_offset), dtype=torch.uint8, device='cuda')
        big[:, :, pitch_offset:] = t
        t = big[:, :, pitch_offset:]
    g = None if gross is None else torch.as_tensor(gross).cuda()
    out = cor.correlate(t, gross=g, surfaces=True)
    o = oracle.correlate(h, w, down, across, frames[0], frames[1:], gross, window=window, search=search, mode='f64',
                         surfaces=True)
    return out, o


@pytest.mark.parametrize('window,search', [(3, 1), (11, 8), (32, 16), (64, 48), (45, 60), (64, 64), (128, 64),
                                           (100, 10)])
def test_surfaces_geometries(window, search):
    h, w = 420, 560
    frames = synth.video(h, w, 3, np.array([[0.0, 0.0], [1.3, -2.2], [-3.6, 2.9]]), np.zeros(3), sigma=2.0, noise=1.0,
                         seed=window * 7 + search)
    out, o = surfaces_vs_oracle(h, w, window, search, frames, skip=max(8, window // 2))
    s = out['surface'].cpu().numpy()
    assert np.abs(s - o['surface']).max() < 2e-6
    d = np.abs(out['offsets'].cpu().numpy() - o['offsets64'])
    assert np.array_equal(np.isnan(d), np.isnan(o['offsets64']))
    if np.isfinite(d).any():
        assert np.nanmax(d) < 1e-4


def test_unaligned_frames_and_per_window_gross():
    h, w = 240, 330
    frames = synth.video(h, w, 4, np.array([[0.0, 0.0], [2.1, 1.2], [-1.4, 3.3], [0.6, -2.7]]), np.zeros(4),
                         sigma=1.5, noise=2.0, seed=5)
    down, across = framecor.window_grid(h, w, 32, 20, 20)
    rng = np.random.default_rng(9)
    gross = rng.integers(-3, 4, (3, len(down[:3]), len(across[:4]), 2)).astype(np.int32)
    out, o = surfaces_vs_oracle(h, w, 32, 20, frames, gross=gross, skip=20, pitch_offset=5)
    assert np.abs(out['surface'].cpu().numpy() - o['surface']).max() < 2e-6
    d = np.abs(out['offsets'].cpu().numpy() - o['offsets64'])
    assert np.array_equal(np.isnan(d), np.isnan(o['offsets64']))
    assert np.nanmax(d) < 1e-4


def test_many_launches_host_path():
    """More frames than one launch: the same outputs one frame at a time."""
    frames, motion, step = synth.small(n=40, h=180, w=320)
    down, across = framecor.window_grid(180, 320, 32, 16, 16)
    cor = framecor.Correlator(180, 320, down, across, window=32, search=16, backend='b200')
    cor.set_form('int8')
    cor.set_reference(frames[0])
    all_at_once = cor.correlate(frames)
    for k in (0, 17, 39):
        one = cor.correlate(frames[k:k + 1])
        for key in one:
            assert np.array_equal(one[key][0], all_at_once[key][k], equal_nan=True), (k, key)


def test_matches_fft32_on_hd():
    """720p, window 64, search 48: both forms agree to the FP32 form's own rounding."""
    c = cases.case('hd')
    cor = correlator(c, 'fft32')
    f, g = torch.as_tensor(c['frames']).cuda(), torch.as_tensor(c['gross']).cuda()
    s32 = cor.correlate(f, gross=g, surfaces=True)['surface']
    cor.set_form('int8')
    s8 = cor.correlate(f, gross=g, surfaces=True)['surface']
    assert (s8 - s32).abs().max().item() < 2e-5


def test_form_limits():
    down, across = framecor.window_grid(600, 600, 200, 20, 100)   # window beyond the int32 bound
    cor = framecor.Correlator(600, 600, down, across, window=200, search=20, backend='b200')
    with pytest.raises(ValueError, match='exact tensor-core'):
        cor.set_form('int8')
