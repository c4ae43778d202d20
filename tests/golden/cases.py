"""
The golden cases: seeded inputs for framecor's correlate, regenerated identically wherever the
same numpy runs (each fixture stores a sha256 of its inputs to prove it). The outputs in
tests/golden/*.npz come from the reference's own CPU backend (make_golden.py).

Each case: frame size, window grid, window, search, stat_size, the reference frame, the frames
and the gross offsets (None, per frame (n, 2) or per window (n, ny, nx, 2)).
"""

import hashlib

import numpy as np

from slipcam_b200 import synth
from slipcam_b200.framecor import window_grid


def _moved(h, w, motion, *, sigma=2.0, noise=1.0, seed=0, step=None, angle=None):
    """Frame 0 at rest (the reference) followed by one frame per motion."""
    motion = np.concatenate([[[0.0, 0.0]], np.asarray(motion, float)])
    step = np.zeros(len(motion)) if step is None else np.concatenate([[0.0], step])
    v = synth.video(h, w, len(motion), motion, step, sigma=sigma, noise=noise, seed=seed, angle=angle)
    return v[0], v[1:]


def case(name):
    """The inputs of a golden case, a dict."""
    stat = 21
    gross = None
    if name == 'shifts':          # known shifts, the reference test's geometry (L = 80)
        h, w, W, R, skip, margin = 240, 320, 32, 24, 24, 0
        ref, frames = _moved(h, w, [(0, 0), (0.3, -0.7), (5.25, -12.5), (-20.4, 15.1)], seed=10)
    elif name == 'gross':         # motion beyond the search range, per-frame gross (L = 44)
        h, w, W, R, skip, margin = 240, 320, 32, 6, 16, 32
        ref, frames = _moved(h, w, [(30.4, -27.6), (30.4, -27.6)], seed=11)
        gross = np.array([[30, -28], [0, 0]], np.int32)
    elif name == 'window_gross':  # per-window gross, odd sizes (L = 27), w not a multiple of 16
        h, w, W, R, skip, margin = 100, 150, 17, 5, 9, 6
        ref, frames = _moved(h, w, [(1.3, -2.2), (-3.7, 0.4), (0.1, 4.9)], seed=12, sigma=1.5)
        down, across = window_grid(h, w, W, R, skip, margin)
        rng = np.random.default_rng(5)
        gross = rng.integers(-6, 7, size=(3, len(down), len(across), 2)).astype(np.int32)
        stat = 5
    elif name == 'invalid':       # outside the frame, and flat reference windows
        h, w, W, R, skip, margin = 240, 320, 32, 24, 24, 0
        ref, frames = _moved(h, w, [(0.0, 0.0), (2.5, 1.5)], seed=13)
        ref = ref.copy()
        ref[:120] = 100
        gross = np.array([[0, 1000], [0, 0]], np.int32)
    elif name == 'small':         # the small workload, 4 of its frames (L = 64)
        h, w, W, R, skip, margin = 360, 640, 32, 16, 16, 0
        v, _, _ = synth.small(n=16)
        ref, frames = v[0], v[[1, 5, 10, 15]]
    elif name == 'hd':            # the 720p workload's geometry (L = 160), 2 frames
        h, w, W, R, skip, margin = 720, 1280, 64, 48, 16, 0
        motion = [(3.2, -4.7), (-6.6, 2.3)]
        ref, frames = _moved(h, w, motion, seed=14, noise=2.0, step=np.array([0.0, 21.5]), angle=30.0)
        gross = np.rint(np.array(motion)).astype(np.int32)
    elif name == 'wide':          # search 64 (L = 192), window 64
        h, w, W, R, skip, margin = 384, 512, 64, 64, 48, 0
        ref, frames = _moved(h, w, [(7.3, -11.6)], seed=15, noise=3.0)
    elif name == 'big':           # window 128, search 64 (L = 256)
        h, w, W, R, skip, margin = 400, 480, 128, 64, 40, 0
        ref, frames = _moved(h, w, [(-9.4, 13.2)], seed=16)
    elif name == 'mixed':         # flat, saturated and striped regions (near-tie peaks)
        h, w, W, R, skip, margin = 256, 384, 32, 16, 16, 0
        v, _ = synth.mixed(n=3, h=h, w=w)
        ref, frames = v[0], v[1:]
        rng = np.random.default_rng(7)
        down, across = window_grid(h, w, W, R, skip, margin)
        gross = rng.integers(-8, 9, size=(2, len(down), len(across), 2)).astype(np.int32)
    elif name in C3:              # a 2-frame slice of the mixed-grid 720p workload (10 % flat, 5 %
        # saturated, an 8 px striped box), one of its three grids, per-window gross U[-20, 20]
        h, w, skip, margin = 720, 1280, 16, 0
        W, R = C3[name]
        v, _ = synth.mixed(n=3, h=h, w=w)
        ref, frames = v[0], v[1:]
        rng = np.random.default_rng(W)
        down, across = window_grid(h, w, W, R, skip, margin)
        gross = rng.integers(-20, 21, size=(2, len(down), len(across), 2)).astype(np.int32)
    else:
        raise KeyError(name)
    down, across = window_grid(h, w, W, R, skip, margin)
    return dict(name=name, height=h, width=w, down=np.asarray(down), across=np.asarray(across),
                window=W, search=R, stat_size=stat, reference=np.ascontiguousarray(ref),
                frames=np.ascontiguousarray(frames), gross=gross)


C3 = {'c3_w32': (32, 16), 'c3_w64': (64, 48), 'c3_w128': (128, 64)}
NAMES = ['shifts', 'gross', 'window_gross', 'invalid', 'small', 'hd', 'wide', 'big', 'mixed', *C3]
# the large cases, checked against the FP64 oracle on a sub-grid (every a-th row, b-th column)
SUBGRID = {'hd': (7, 9), 'c3_w32': (7, 9), 'c3_w64': (7, 9), 'c3_w128': (5, 9)}


def digest(c):
    """A sha256 of a case's inputs."""
    m = hashlib.sha256()
    for key in ('reference', 'frames', 'down', 'across'):
        m.update(np.ascontiguousarray(c[key]).tobytes())
    if c['gross'] is not None:
        m.update(np.ascontiguousarray(c['gross'], np.int32).tobytes())
    m.update(repr((c['height'], c['width'], c['window'], c['search'], c['stat_size'])).encode())
    return m.hexdigest()

