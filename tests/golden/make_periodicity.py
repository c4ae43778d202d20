"""
Golden vectors of auto_slip.periodicity (python/slipcam/auto_slip.py:105-129): the reference
function itself, taken from the reference's source file by its name (its module imports matplotlib,
which is not installed) and run with numpy and scipy on seeded synthetic reference frames. Writes
tests/golden/periodicity.npz. Run here, where the reference is mounted:

    python tests/golden/make_periodicity.py /root/reference
"""

import ast
import os
import sys

import numpy as np
from scipy import ndimage, signal

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from slipcam_b200 import synth   # noqa: E402


def reference_periodicity(root):
    path = os.path.join(root, 'python', 'slipcam', 'auto_slip.py')
    tree = ast.parse(open(path).read())
    fn = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == 'periodicity')
    ns = {'np': np, 'signal': signal, 'ndimage': ndimage}
    exec(compile(ast.Module(body=[fn], type_ignores=[]), path, 'exec'), ns)
    return ns['periodicity']


def frame(seed):
    """A textured frame with a periodic stripe box (8 px) and a flat box, uint8."""
    rng = np.random.default_rng(seed)
    h, w = 176, 240
    f = synth.texture(h, w, 1.5, rng)
    f[20:90, 130:230] = 128 + 60 * np.sin(2 * np.pi * np.arange(100) / 8.0)[None, :]
    f[110:170, 10:80] = 100
    return np.clip(np.rint(f), 0, 255).astype(np.uint8)


def main(root):
    per = reference_periodicity(root)
    cases = {}
    for k, (window, search, skip) in enumerate([(32, 12, 16), (24, 8, 20)]):
        ref = frame(40 + k)
        h, w = ref.shape
        first = search
        y0 = np.arange(first, h - search - window + 1, skip)
        x0 = np.arange(first, w - search - window + 1, skip)
        out = per(ref, y0, x0, window, search)
        cases.update({f'ref{k}': ref, f'y0{k}': y0, f'x0{k}': x0, f'out{k}': out,
                      f'geom{k}': np.array([window, search, 5])})
    np.savez(os.path.join(HERE, 'periodicity.npz'), **cases)
    print('wrote periodicity.npz', {k: v.shape for k, v in cases.items() if k.startswith('out')})


if __name__ == '__main__':
    main(sys.argv[1] if len(sys.argv) > 1 else '/root/reference')
