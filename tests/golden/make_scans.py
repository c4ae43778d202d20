"""
Golden vectors of auto_slip.frame_differences and auto_slip.text_mask (python/slipcam/auto_slip.py:
56-94): the reference functions themselves, taken from the reference's source by name (the module
imports matplotlib, which is not installed) and run with numpy and scipy on a seeded synthetic
video with burned-in text. Writes tests/golden/scans.npz. Run here, where the reference is mounted:

    python tests/golden/make_scans.py /root/reference
"""

import ast
import os
import sys

import numpy as np
from scipy import ndimage

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from slipcam_b200 import synth   # noqa: E402


def reference_functions(root):
    path = os.path.join(root, 'python', 'slipcam', 'auto_slip.py')
    tree = ast.parse(open(path).read())
    fns = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in ('frame_differences', 'text_mask')]
    ns = {'np': np, 'ndimage': ndimage}
    exec(compile(ast.Module(body=fns, type_ignores=[]), path, 'exec'), ns)
    return ns['frame_differences'], ns['text_mask']


def video(seed=5, n=48, h=120, w=168):
    """A shaking texture with fixed burned-in text: glyph strokes and a caption box outline."""
    rng = np.random.default_rng(seed)
    mover = synth.Mover(synth.texture(h, w, 2.0, rng))
    motion = np.cumsum(rng.normal(0, 0.8, (n, 2)), 0)
    motion[:4] = 0   # a short freeze at the start
    frames = np.empty((n, h, w), np.uint8)
    for k in range(n):
        img = mover.shifted(*motion[k]) + rng.standard_normal((h, w)) * 1.5
        img[8:12, 10:70] = 250                      # strokes of a clock
        img[8:24, 10:13] = 250
        img[16:20, 30:60] = 20
        img[90:112, 100:160] = 30                   # a caption box with a bright outline
        img[90:92, 100:160] = img[110:112, 100:160] = 240
        img[90:112, 100:102] = img[90:112, 158:160] = 240
        frames[k] = np.clip(np.rint(img), 0, 255)
    return frames


def main(root):
    fd, tm = reference_functions(root)
    v = video()
    d = fd(v, chunk=20)
    mask = tm(v, 4, nframes=40, chunk=10)
    mask2 = tm(v, 6, nframes=30, chunk=6, edge_percentile=85, max_std=2.0, dilate=2)
    mask0 = tm(v, 6, nframes=30, chunk=6, edge_percentile=85, max_std=2.0, dilate=0)   # dilation until no change
    np.savez(os.path.join(HERE, 'scans.npz'), frames=v, diff=d, mask=mask, mask2=mask2, mask0=mask0)
    print('wrote scans.npz', d.shape, mask.sum(), mask2.sum())


if __name__ == '__main__':
    main(sys.argv[1] if len(sys.argv) > 1 else '/root/reference')
