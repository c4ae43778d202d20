"""
Golden vectors of stabilize.coarse_track, stabilize.ncc_peak, stabilize.warp and stabilize.stabilize
(python/slipcam/stabilize.py:22-124, with slip_series.fit_camera, python/slipcam/slip_series.py:49-72):
the reference functions
themselves, taken from the reference's source by name (slip_series imports matplotlib, which is not
installed) and run with numpy and scipy on seeded synthetic videos of a moving camera
(slipcam_b200.synth.camera). Writes tests/golden/stabilize.npz. Run here, where the reference is
mounted:

    python tests/golden/make_stabilize.py /root/reference
"""

import ast
import os
import sys

import numpy as np
from scipy import ndimage, signal

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from slipcam_b200 import synth   # noqa: E402


def _functions(path, names, ns):
    tree = ast.parse(open(path).read())
    fns = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names]
    exec(compile(ast.Module(body=fns, type_ignores=[]), path, 'exec'), ns)
    return [ns[n] for n in names]


def reference_functions(root):
    py = os.path.join(root, 'python', 'slipcam')
    ns = {'np': np, 'ndimage': ndimage, 'signal': signal}
    _functions(os.path.join(py, 'slip_series.py'), ['fit_camera'], ns)
    fns = _functions(os.path.join(py, 'stabilize.py'), ['ncc_peak', 'apply', 'coarse_track', 'warp', 'stabilize'], ns)
    return fns[0], fns[2], ns['fit_camera'], fns[3], fns[4]


def main(root):
    ncc_peak, coarse_track, fit_camera, warp, stabilize = reference_functions(root)
    out = {}
    # a small grid: 48-px windows 40 px apart, +-12 px search; a flat patch, text, a blank frame
    f, p, m = synth.camera(12, 240, 320, ref=4, seed=6, flat=(236, 150, 300, 232), blank=(9,))
    params, used, count = coarse_track(f, 4, m, window=48, step=40, search=12, start=1)
    out.update(a_frames=f, a_text=m, a_truth=p, a_params=params, a_used=used, a_count=count)
    # the reference's defaults (96-px windows, 96 apart, +-32 px) on 360 x 480 frames, larger steps
    f, p, m = synth.camera(8, 360, 480, ref=2, seed=8, walk=(6.0, 6.0, 0.004, 0.004), text=((300, 300, 460, 340),))
    params, used, count = coarse_track(f, 2, m)
    out.update(b_frames=f, b_text=m, b_truth=p, b_params=params, b_used=used, b_count=count)
    # ncc_peak alone: a template cut from a frame and searched in the next, a peak on the border,
    # a flat template, a flat search window
    rng = np.random.default_rng(9)
    img = synth.texture(200, 200, 2.0, rng)
    cases = [(img[50:98, 60:108], img[42:110, 49:117]),     # the template 8 / 11 px in: off centre
             (img[50:98, 60:108], img[50:118, 60:128]),     # the match at the first placement (a border)
             (np.full((48, 48), 7.0), img[0:68, 0:68]),     # a flat template
             (img[10:58, 10:58], np.full((68, 68), 90.0)),  # a flat search window
             (img[100:132, 120:152] + rng.normal(0, 3, (32, 32)), img[90:150, 105:165])]
    out['ncc_templates'] = np.array([c[0] for c in cases[:4]])
    out['ncc_searches'] = np.array([c[1] for c in cases[:4]])
    out['ncc_t5'], out['ncc_s5'] = cases[4]
    out['ncc_out'] = np.array([ncc_peak(t, s) for t, s in cases])
    # fit_camera alone: a transform, noise, and gross outliers
    x = rng.uniform(-300, 300, 40)
    y = rng.uniform(-200, 200, 40)
    truth = np.array([3.0, -2.0, 0.01, -0.005])
    dx = truth[0] - truth[2] * y + truth[3] * x + rng.normal(0, 0.05, 40)
    dy = truth[1] + truth[2] * x + truth[3] * y + rng.normal(0, 0.05, 40)
    dx[:5] += 7.0
    dy[5:8] -= 4.0
    dx[8:10] = np.nan
    fit, nfit = fit_camera(dx, dy, x, y)
    out.update(fit_dx=dx, fit_dy=dy, fit_x=x, fit_y=y, fit=fit, fit_used=nfit)
    # warp and stabilize: case a's frames onto its reference with its transforms (frame 0 has none)
    f, text = out['a_frames'][1:], out['a_text']
    stab, union = stabilize(f, out['a_params'][1:], text)
    out.update(stab_out=stab, stab_union=union)
    # a thick text box (its middle more than 15 px from any pixel without text: the mean fills it)
    thick = np.zeros_like(text)
    thick[100:150, 60:200] = True
    stab2, union2 = stabilize(f[:4], out['a_params'][1:5], thick)
    out.update(stab2_text=thick, stab2_out=stab2, stab2_union=union2)
    frame = out['b_frames'][3].astype(np.float32)
    out.update(warp_params=np.array([3.3, -7.6, 0.012, -0.008]), warp_frame=frame)
    out['warp_out'] = warp(frame, out['warp_params'])
    out['warp_out_fill'] = warp(frame, out['warp_params'], fill=17.25)
    np.savez_compressed(os.path.join(HERE, 'stabilize.npz'), **out)
    print('wrote stabilize.npz', out['a_used'], out['b_used'], out['ncc_out'], fit, nfit)


if __name__ == '__main__':
    main(sys.argv[1] if len(sys.argv) > 1 else '/root/reference')
