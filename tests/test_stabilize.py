"""
stabilize.coarse_track / ncc_peak (python/slipcam/stabilize.py:22-96, slip_series.fit_camera
python/slipcam/slip_series.py:49-72) on the b200 backend.

CPU: the oracle against the reference's golden vectors (tests/golden/make_stabilize.py), host logic.
GPU: the peak kernel against the same epilogue in numpy on the same float32 surfaces; the fit kernel
against the oracle's fit; coarse_track against the golden vectors and the oracle, at small sizes and
at 720p with the reference's defaults (96-px windows, +-32 px), and against the true motion.

Tolerances: the GPU correlates in FP32 where the reference works in float64, so the peak positions
differ by ~1e-5 px; the transforms are compared to 2e-3 px (p, q) and 1e-5 (a, s).
"""

import ctypes
import os

import numpy as np
import pytest

from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, 'golden', 'stabilize.npz'))
TOL = np.array([2e-3, 2e-3, 1e-5, 1e-5])


def _same_transforms(a, b, tol=TOL):
    assert np.array_equal(np.isnan(a), np.isnan(b))
    ok = ~np.isnan(a[:, 0])
    assert np.all(np.abs(a[ok] - b[ok]) <= tol), np.abs(a[ok] - b[ok]).max(0)


# ---- CPU: the oracle pinned to the reference ----

def test_oracle_ncc_peak_golden():
    out = [oracle.ncc_peak(t, s) for t, s in zip(GOLD['ncc_templates'], GOLD['ncc_searches'])]
    out.append(oracle.ncc_peak(GOLD['ncc_t5'], GOLD['ncc_s5']))
    out, ref = np.array(out), GOLD['ncc_out']
    for k in (0, 1, 4):
        np.testing.assert_allclose(out[k], ref[k], rtol=0, atol=1e-9)
    assert np.isnan(out[2, :2]).all() and out[2, 2] == 0 == ref[2, 2]   # a flat template
    # a flat search window: the correlation is rounding noise; its position is not defined
    assert abs(out[3, 2]) < 1e-6 and abs(ref[3, 2]) < 1e-6


def test_oracle_fit_camera_golden():
    fit, n = oracle.fit_camera(GOLD['fit_dx'], GOLD['fit_dy'], GOLD['fit_x'], GOLD['fit_y'])
    np.testing.assert_allclose(fit, GOLD['fit'], rtol=0, atol=1e-9)
    assert n == GOLD['fit_used']


def test_oracle_fit_camera_too_few():
    x = np.array([0.0, 10.0, 20.0, 30.0])
    fit, n = oracle.fit_camera(np.array([1.0, 1.0, np.nan, 1.0]), np.zeros(4), x, x)
    assert np.isnan(fit).all() and n == 0


@pytest.mark.parametrize('case', ['a', 'b'])
def test_oracle_coarse_track_golden(case):
    kw = dict(window=48, step=40, search=12, start=1) if case == 'a' else {}
    ref = 4 if case == 'a' else 2
    params, used, count = oracle.coarse_track(GOLD[case + '_frames'], ref, GOLD[case + '_text'], **kw)
    _same_transforms(params, GOLD[case + '_params'], np.full(4, 1e-9))
    assert np.array_equal(used, GOLD[case + '_used']) and count == GOLD[case + '_count']


def test_apply_matches_formula():
    from slipcam_b200 import stabilize
    x, y = np.array([-100.0, 5.0]), np.array([40.0, -60.0])
    p = (1.5, -2.0, 0.01, -0.02)
    ax, ay = stabilize.apply(p, x, y)
    np.testing.assert_array_equal(ax, x + 1.5 - 0.01 * y + -0.02 * x)
    np.testing.assert_array_equal(ay, y + -2.0 + 0.01 * x + -0.02 * y)


def test_template_grid_and_keep():
    from slipcam_b200 import stabilize
    yc, xc = stabilize.template_grid(240, 320, 48, 40, 12)
    np.testing.assert_array_equal(yc, np.arange(36, 204, 40))
    np.testing.assert_array_equal(xc, np.arange(36, 284, 40))
    keep = stabilize._keep(GOLD['a_frames'][4], GOLD['a_text'], yc, xc, 24)
    assert keep.sum() == GOLD['a_count']


def test_odd_window_rejected():
    from slipcam_b200 import stabilize
    with pytest.raises(ValueError):
        stabilize.coarse_track(np.zeros((2, 64, 64), np.uint8), 0, np.zeros((64, 64), bool), window=31)


def test_entry_points_declared():
    from slipcam_b200 import _lib
    hdr = open(os.path.join(os.path.dirname(HERE), 'include', 'slipcam_b200.h')).read()
    for name in ('b200_ncc_peaks_device', 'b200_coarse_fit_device'):
        assert name in hdr and name in _lib.SIGNATURES
    assert f'#define B200_COARSE_MAX_WINDOWS {_lib.COARSE_MAX_WINDOWS}' in hdr


# ---- GPU ----

def _numpy_peak(s):
    """ncc_peak's epilogue (stabilize.py:35-44) on one float32 surface, in float64"""
    M = s.shape[0]
    i, j = np.unravel_index(int(np.argmax(s)), s.shape)
    c = float(s[i, j])

    def vertex(m, p):
        den = m - 2 * c + p
        return 0.0 if abs(den) < 1e-12 else 0.5 * (m - p) / den
    di = vertex(float(s[i - 1, j]), float(s[i + 1, j])) if 0 < i < M - 1 else 0.0
    dj = vertex(float(s[i, j - 1]), float(s[i, j + 1])) if 0 < j < M - 1 else 0.0
    return i + di - (M - 1) / 2, j + dj - (M - 1) / 2, c


@pytest.mark.gpu
def test_ncc_peaks_kernel():
    import torch
    from slipcam_b200 import stabilize
    rng = np.random.default_rng(3)
    M = 25
    surf = rng.uniform(-0.5, 0.6, (40, M, M)).astype(np.float32)
    yy, xx = np.mgrid[0:M, 0:M]
    for k in range(30):   # smooth peaks, some on the border, some with exact ties
        cy, cx = rng.uniform(-1, M, 2)
        surf[k] = (0.9 - 0.01 * ((yy - cy) ** 2 + (xx - cx) ** 2)).astype(np.float32)
    surf[30] = 0.25                          # all equal: the first
    surf[31, 3, 4] = surf[31, 7, 2] = 2.0    # a tie: the first in raster order
    surf[32, 0, 0] = 3.0                     # a corner
    surf[33, M - 1, 5] = 3.0
    out = stabilize.ncc_peaks(torch.as_tensor(surf).cuda()).cpu().numpy()
    ref = np.array([_numpy_peak(s) for s in surf])
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12)
    empty = stabilize.ncc_peaks(torch.empty((0, M, M), device='cuda'))
    assert empty.shape == (0, 3)


def _fit_on_gpu(dx, dy, yc, xc, h, w, keep, min_peak=0.5, peak=None):
    """the fit kernel on offsets given as peaks with zero gross; returns (params, used, next gross, prev)"""
    import torch
    from slipcam_b200 import _lib
    ny, nx = len(yc), len(xc)
    nwin = ny * nx
    peaks = np.zeros((nwin, 3))
    peaks[:, 0], peaks[:, 1] = dy, dx
    peaks[:, 2] = 1.0 if peak is None else peak
    d = lambda a, t: torch.as_tensor(np.ascontiguousarray(a, t)).cuda()
    pk, gross = d(peaks, np.float64), torch.zeros((nwin, 2), dtype=torch.int32, device='cuda')
    keep_d, yc_d, xc_d = d(keep.ravel().astype(np.uint8), np.uint8), d(yc, np.int32), d(xc, np.int32)
    prev = torch.zeros(4, dtype=torch.float64, device='cuda')
    params = torch.full((4,), float('nan'), dtype=torch.float64, device='cuda')
    used = torch.zeros(1, dtype=torch.int32, device='cuda')
    rc = _lib.lib().b200_coarse_fit_device(pk.data_ptr(), gross.data_ptr(), keep_d.data_ptr(), yc_d.data_ptr(),
                                           xc_d.data_ptr(), ny, nx, h, w, 48, 12, ctypes.c_double(min_peak),
                                           prev.data_ptr(), params.data_ptr(), used.data_ptr(),
                                           torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.OK
    return params.cpu().numpy(), int(used.item()), gross.cpu().numpy(), prev.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize('seed', [0, 1, 2])
def test_fit_kernel_matches_oracle(seed):
    from slipcam_b200 import stabilize
    h, w = 480, 640
    yc, xc = stabilize.template_grid(h, w, 48, 40, 12)
    Y, X = np.meshgrid(yc - h / 2, xc - w / 2, indexing='ij')
    rng = np.random.default_rng(seed)
    truth = rng.normal(0, 1, 4) * [3, 3, 0.01, 0.01]
    dx = truth[0] - truth[2] * Y + truth[3] * X + rng.normal(0, 0.08, Y.shape)
    dy = truth[1] + truth[2] * X + truth[3] * Y + rng.normal(0, 0.08, Y.shape)
    bad = rng.random(Y.shape) < 0.15   # outliers, some beyond the 0.3 px floor only a little
    dx[bad] += rng.choice([-1, 1], bad.sum()) * rng.uniform(0.5, 9, bad.sum())
    keep = rng.random(Y.shape) > 0.1
    peak = np.where(rng.random(Y.shape) < 0.05, 0.3, 0.9)   # some below min_peak
    params, used, gross, prev = _fit_on_gpu(dx.ravel(), dy.ravel(), yc, xc, h, w, keep, peak=peak.ravel())
    sel = keep & (peak >= 0.5)
    ref, nref = oracle.fit_camera(np.where(sel, dx, np.nan).ravel(), np.where(sel, dy, np.nan).ravel(), X.ravel(),
                                  Y.ravel())
    np.testing.assert_allclose(params, ref, rtol=0, atol=1e-9)
    assert used == nref
    np.testing.assert_array_equal(prev, params)
    # the next frame's gross offsets: the rounded predicted centres minus the grid's
    px, py = stabilize.apply(params, X.ravel(), Y.ravel())
    np.testing.assert_array_equal(gross[:, 0], np.rint(py + h / 2) - (Y.ravel() + h / 2))
    np.testing.assert_array_equal(gross[:, 1], np.rint(px + w / 2) - (X.ravel() + w / 2))


@pytest.mark.gpu
def test_fit_kernel_too_few_windows():
    from slipcam_b200 import stabilize
    h, w = 240, 320
    yc, xc = stabilize.template_grid(h, w, 48, 40, 12)
    keep = np.zeros((len(yc), len(xc)), bool)
    keep.ravel()[:3] = True
    params, used, gross, prev = _fit_on_gpu(np.ones(keep.size), np.ones(keep.size), yc, xc, h, w, keep)
    assert used == 0 and np.all(params == 0) and np.all(prev == 0) and np.all(gross == 0)


@pytest.mark.gpu
@pytest.mark.parametrize('case', ['a', 'b'])
def test_coarse_track_golden(case):
    from slipcam_b200 import stabilize
    kw = dict(window=48, step=40, search=12, start=1) if case == 'a' else {}
    ref = 4 if case == 'a' else 2
    params, used, count = stabilize.coarse_track(GOLD[case + '_frames'], ref, GOLD[case + '_text'], **kw)
    _same_transforms(params, GOLD[case + '_params'])
    assert np.array_equal(used, GOLD[case + '_used']) and count == GOLD[case + '_count']


@pytest.mark.gpu
def test_coarse_track_device_frames_and_chunks():
    import torch
    from slipcam_b200 import stabilize
    f, text = GOLD['a_frames'], GOLD['a_text']
    kw = dict(window=48, step=40, search=12, start=1)
    a = stabilize.coarse_track(f, 4, text, **kw)
    b = stabilize.coarse_track(torch.as_tensor(f).cuda(), 4, torch.as_tensor(text), **kw)
    c = stabilize.coarse_track(f, 4, text, chunk=3, **kw)   # runs split across chunks, both passes
    for other in (b, c):
        np.testing.assert_array_equal(a[0], other[0])
        np.testing.assert_array_equal(a[1], other[1])


@pytest.mark.gpu
def test_coarse_track_edges():
    from slipcam_b200 import stabilize
    f, text = GOLD['a_frames'], GOLD['a_text']
    kw = dict(window=48, step=40, search=12)
    # the reference as the last frame (no forward pass), as the first (no backward pass)
    for ref in (len(f) - 1, 0):
        p, u, n = stabilize.coarse_track(f, ref, text, **kw)
        po, uo, no = oracle.coarse_track(f, ref, text, **kw)
        _same_transforms(p, po)
        assert np.array_equal(u, uo) and n == no
    # no window fits: the transforms stay zero, no fit anywhere
    p, u, n = stabilize.coarse_track(f[:, :60, :60], 1, text[:60, :60], **kw)
    po, uo, no = oracle.coarse_track(f[:, :60, :60], 1, text[:60, :60], **kw)
    assert np.array_equal(p, po) and np.array_equal(u, uo) and n == no == 0
    # everything under text: no template in use
    p, u, n = stabilize.coarse_track(f[:5], 2, np.ones_like(text), **kw)
    po, uo, no = oracle.coarse_track(f[:5], 2, np.ones_like(text), **kw)
    assert np.array_equal(p, po) and np.array_equal(u, uo) and n == no == 0


@pytest.mark.gpu
def test_coarse_track_720p_defaults():
    """The reference's defaults on 720p frames: against the oracle and the true motion."""
    import torch
    from slipcam_b200 import stabilize, synth
    f, truth, text = synth.camera(10, 720, 1280, ref=3, seed=11, walk=(5.0, 5.0, 0.002, 0.002),
                                  text=((900, 24, 1240, 68), (40, 650, 630, 700)), blank=(7,), device='cuda')
    p, u, n = stabilize.coarse_track(f, 3, text)
    po, uo, no = oracle.coarse_track(f.cpu().numpy(), 3, text)
    _same_transforms(p, po)
    assert np.array_equal(u, uo) and n == no and n > 50
    assert u[7] == 0 and np.array_equal(p[7], p[6])   # the blank frame keeps the previous transform
    good = np.array([k for k in range(10) if k != 7])
    assert np.abs(p[good, :2] - truth[good, :2]).max() < 0.1
    assert np.abs(p[good, 2:] - truth[good, 2:]).max() < 2e-4


@pytest.mark.gpu
def test_coarse_track_long_video_groups():
    """More frames per call than one group of tables (the tables of the next group are built while
    the frames of one are tracked): the same transforms as the oracle, whatever the chunking."""
    import torch
    from slipcam_b200 import stabilize, synth
    f, truth, text = synth.camera(100, 240, 320, ref=30, seed=12, walk=(1.5, 1.5, 0.002, 0.002))
    kw = dict(window=48, step=40, search=12)
    p, u, n = stabilize.coarse_track(f, 30, text, chunk=100, **kw)
    po, uo, no = oracle.coarse_track(f, 30, text, **kw)
    _same_transforms(p, po)
    assert np.array_equal(u, uo) and n == no
    for other in (stabilize.coarse_track(f, 30, text, chunk=7, **kw),
                  stabilize.coarse_track(torch.as_tensor(f).cuda(), 30, text, chunk=70, **kw)):
        np.testing.assert_array_equal(p, other[0])
        np.testing.assert_array_equal(u, other[1])


@pytest.mark.gpu
def test_coarse_track_big_transform():
    """A search window of 256 pixels (window 128, search 64): the big transform's surfaces and the
    separate peak kernel."""
    from slipcam_b200 import stabilize, synth
    f, truth, text = synth.camera(6, 600, 800, ref=2, seed=13, walk=(8.0, 8.0, 0.003, 0.003), text=((20, 540, 300, 580),))
    kw = dict(window=128, step=128, search=64)
    p, u, n = stabilize.coarse_track(f, 2, text, **kw)
    po, uo, no = oracle.coarse_track(f, 2, text, **kw)
    _same_transforms(p, po)
    assert np.array_equal(u, uo) and n == no and n >= 8


# ---- stabilize.warp / stabilize.stabilize (stabilize.py:99-124) ----

def test_oracle_warp_stabilize_golden():
    o, u = oracle.stabilize(GOLD['a_frames'][1:], GOLD['a_params'][1:], GOLD['a_text'])
    assert np.array_equal(o, GOLD['stab_out']) and np.array_equal(u, GOLD['stab_union'])
    o, u = oracle.stabilize(GOLD['a_frames'][1:5], GOLD['a_params'][1:5], GOLD['stab2_text'])
    assert np.array_equal(o, GOLD['stab2_out']) and np.array_equal(u, GOLD['stab2_union'])
    assert np.array_equal(oracle.warp(GOLD['warp_frame'], GOLD['warp_params']), GOLD['warp_out'])
    assert np.array_equal(oracle.warp(GOLD['warp_frame'], GOLD['warp_params'], 17.25), GOLD['warp_out_fill'])


def test_oracle_box_mean_matches_definition():
    """the box mean against a direct window average with the half-sample reflection (small case)"""
    rng = np.random.default_rng(2)
    x = rng.integers(0, 256, (13, 17)).astype(np.float32)
    size = 5

    def reflect(i, n):
        i %= 2 * n
        return i if i < n else 2 * n - 1 - i
    a = np.array([[np.mean([x[reflect(r + k, 13), c] for k in range(-2, 3)]) for c in range(17)] for r in range(13)],
                 np.float32)
    b = np.array([[np.mean([a[r, reflect(c + k, 17)] for k in range(-2, 3)], dtype=np.float64) for c in range(17)]
                  for r in range(13)]).astype(np.float32)
    np.testing.assert_allclose(oracle.box_mean(x, size), b, rtol=1e-6)


def _diff_stats(a, b):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    return int(d.max()) if d.size else 0, int((d > 0).sum())


@pytest.mark.gpu
def test_stabilize_golden():
    """The GPU against the reference's own outputs: bit-identical frames and text union."""
    from slipcam_b200 import stabilize
    o, u = stabilize.stabilize(GOLD['a_frames'][1:], GOLD['a_params'][1:], GOLD['a_text'])
    assert _diff_stats(o, GOLD['stab_out']) == (0, 0)
    assert np.array_equal(u, GOLD['stab_union'])
    o, u = stabilize.stabilize(GOLD['a_frames'][1:5], GOLD['a_params'][1:5], GOLD['stab2_text'])
    assert _diff_stats(o, GOLD['stab2_out']) == (0, 0)
    assert np.array_equal(u, GOLD['stab2_union'])


@pytest.mark.gpu
def test_warp_golden():
    from slipcam_b200 import stabilize
    np.testing.assert_array_equal(stabilize.warp(GOLD['warp_frame'], GOLD['warp_params']), GOLD['warp_out'])
    np.testing.assert_array_equal(stabilize.warp(GOLD['warp_frame'], GOLD['warp_params'], fill=17.25),
                                  GOLD['warp_out_fill'])


@pytest.mark.gpu
def test_stabilize_edges():
    """no text at all; device frames; chunks; frames with NaN transforms (fill everywhere)"""
    import torch
    from slipcam_b200 import stabilize
    f, p = GOLD['a_frames'][1:7], GOLD['a_params'][1:7].copy()
    none = np.zeros_like(GOLD['a_text'])
    o, u = stabilize.stabilize(f, p, none)
    oo, uo = oracle.stabilize(f, p, none)
    assert np.array_equal(o, oo) and not u.any() and not uo.any()
    a = stabilize.stabilize(f, p, GOLD['a_text'])
    b = stabilize.stabilize(torch.as_tensor(f).cuda(), torch.as_tensor(p), GOLD['a_text'])
    c = stabilize.stabilize(f, p, GOLD['a_text'], chunk=4)
    for other in (b, c):
        assert np.array_equal(a[0], np.asarray(other[0].cpu() if hasattr(other[0], 'cpu') else other[0]))
        assert np.array_equal(a[1], np.asarray(other[1].cpu() if hasattr(other[1], 'cpu') else other[1]))
    p[2] = np.nan
    o, u = stabilize.stabilize(f, p, GOLD['a_text'])
    oo, uo = oracle.stabilize(f, p, GOLD['a_text'])
    assert np.array_equal(o, oo) and np.array_equal(u, uo)


@pytest.mark.gpu
def test_stabilize_720p():
    """720p frames with their true transforms: against the oracle, and the warped frames back on the
    reference away from the text and the borders."""
    from slipcam_b200 import stabilize, synth
    boxes = ((900, 24, 1240, 68), (40, 650, 630, 700))
    f, truth, text = synth.camera(4, 720, 1280, ref=0, seed=14, walk=(3.0, 3.0, 0.002, 0.002), text=boxes, noise=0.0)
    o, u = stabilize.stabilize(f, truth, text)
    oo, uo = oracle.stabilize(f, truth, text)
    assert _diff_stats(o, oo) == (0, 0)
    assert np.array_equal(u, uo)
    inner = np.zeros((720, 1280), bool)
    inner[80:600, 80:1200] = True
    inner &= ~text
    err = np.abs(o[1:].astype(np.int32) - f[0].astype(np.int32))[:, inner]
    assert np.median(err) <= 1 and np.percentile(err, 99) <= 6


@pytest.mark.gpu
def test_coarse_track_on_a_side_stream():
    """The library runs the frame chain on its own stream, ordered by events after the caller's work
    and before the caller's next: the same transforms from a non-default torch stream, with the
    frames produced on that stream just before the call."""
    import torch
    from slipcam_b200 import stabilize
    f, text = GOLD['a_frames'], GOLD['a_text']
    kw = dict(window=48, step=40, search=12, start=1)
    a = stabilize.coarse_track(f, 4, text, **kw)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        fd = torch.as_tensor(f).cuda(non_blocking=False) + 0   # produced on the side stream
        tr = stabilize.CoarseTracker(fd[4], text, window=48, step=40, search=12)
        b = tr.run(fd, 4, start=1)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
