"""
Several window grids in one persistent launch (framecor.MultiCorrelator, b200_group_*): every
grid's outputs are those of its own Correlator, bit for bit (the same per-pair device code), with
and without the CUDA graph, after the autotuner, and on new frames in the same buffers.
"""

import numpy as np
import pytest

from slipcam_b200 import framecor, synth

torch = pytest.importorskip('torch')

H, W = 400, 480
GRIDS = [dict(window=32, search=16, skip=24), dict(window=64, search=48, skip=40), dict(window=128, search=64, skip=56)]


def grids():
    out = []
    for g in GRIDS:
        down, across = framecor.window_grid(H, W, g['window'], g['search'], g['skip'])
        out.append(dict(down=down, across=across, window=g['window'], search=g['search']))
    return out


def frames_and_gross(n=3, seed=0):
    v, _ = synth.mixed(n=n + 1, h=H, w=W, seed=seed)
    rng = np.random.default_rng(seed + 5)
    gross = []
    for g in grids():
        gross.append(rng.integers(-20, 21, (n, len(g['down']), len(g['across']), 2)).astype(np.int32))
    gross[0] = None   # one grid without gross, one per window, one per frame
    gross[2] = rng.integers(-6, 7, (n, 2)).astype(np.int32)
    return v[0], v[1:], gross


def singles(ref, frames, gross):
    out = []
    for g, gg in zip(grids(), gross):
        c = framecor.Correlator(H, W, g['down'], g['across'], window=g['window'], search=g['search'], backend='b200')
        c.set_form('fft32')   # the group's arithmetic
        c.set_reference(ref)
        out.append(c.correlate(torch.as_tensor(frames).cuda(), gross=None if gg is None else torch.as_tensor(gg).cuda()))
    return out


def same(a, b):
    for k in ('offsets', 'peak', 'snr', 'cov'):
        x, y = a[k].cpu().numpy(), b[k].cpu().numpy()
        assert np.array_equal(np.isnan(x), np.isnan(y)), k
        assert np.array_equal(x[~np.isnan(x)], y[~np.isnan(y)]), (k, np.nanmax(np.abs(x - y)))


@pytest.mark.gpu
def test_group_matches_each_correlator():
    ref, frames, gross = frames_and_gross()
    mc = framecor.MultiCorrelator(H, W, grids())
    mc.set_reference(ref)
    assert [c.info()[2] for c in mc.grids] == [64, 160, 256]
    got = mc.correlate(torch.as_tensor(frames).cuda(), gross=[None if g is None else torch.as_tensor(g) for g in gross])
    want = singles(ref, frames, gross)
    for a, b in zip(got, want):
        same(a, b)
        assert np.isfinite(a['offsets'].cpu().numpy()).mean() > 0.3


@pytest.mark.gpu
def test_group_graph_replay_and_configs():
    ref, frames, gross = frames_and_gross(seed=1)
    ref2, frames2, _ = frames_and_gross(seed=2)
    mc = framecor.MultiCorrelator(H, W, grids())
    mc.set_reference(ref)
    buf = torch.as_tensor(frames).cuda()
    g = [None if x is None else torch.as_tensor(x).cuda() for x in gross]
    first = mc.correlate(buf, gross=g)
    buf.copy_(torch.as_tensor(frames2))           # new frames in the same buffer: the graph replays
    second = mc.correlate(buf, gross=g)
    want2 = singles(ref, frames2, gross)
    for a, b in zip(second, want2):
        same(a, b)
    for cfg in (dict(threads=512, chunk=4, costly_first=False, graph=False), dict(threads=256, chunk=8, graph=True),
                dict(per_grid=True, graph=True), dict(per_grid=True, graph=False)):
        mc.set_config(**cfg)
        buf.copy_(torch.as_tensor(frames))
        again = mc.correlate(buf, gross=g)
        for a, b in zip(again, first):
            same(a, b)


@pytest.mark.gpu
def test_group_autotuner():
    ref, frames, gross = frames_and_gross(seed=3)
    mc = framecor.MultiCorrelator(H, W, grids())
    mc.set_reference(ref)
    f = torch.as_tensor(frames).cuda()
    g = [None if x is None else torch.as_tensor(x).cuda() for x in gross]
    ms, cfg = mc.tune(f, gross=g)
    assert ms > 0 and cfg['threads'] in (256, 512) and cfg['chunk'] in (1, 2, 4, 8)
    for a, b in zip(mc.correlate(f, gross=g), singles(ref, frames, gross)):
        same(a, b)


@pytest.mark.gpu
def test_group_errors():
    g = grids()
    with pytest.raises(ValueError, match='1 to 4'):
        framecor.MultiCorrelator(H, W, g * 2)
    mc = framecor.MultiCorrelator(H, W, g[:2])
    with pytest.raises(RuntimeError, match='set_reference'):
        mc.correlate(torch.zeros((1, H, W), dtype=torch.uint8, device='cuda'))
    with pytest.raises(ValueError, match='CUDA frames'):
        mc.correlate(np.zeros((1, H, W), np.uint8))
