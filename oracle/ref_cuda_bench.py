"""
TEST INFRASTRUCTURE: a baseline, never the product. The reference's own CUDA backend (slipcam
cxx/cuda.cu: cuFFT R2C / C2R batches with its extract, multiplyConjugate, normalize and peaks
kernels), built unchanged for sm_100a by oracle/Makefile (target ref_cuda) into oracle/_ref/cuda,
timed through the reference's own Python API on the 720p workload (720 x 1280 frames, window 64,
search 48, skip 16: 2450 windows per frame, per-frame gross offsets, 16 frames per call) or the
1080p streaming one (1080 x 1920, window 64, search 64, skip 8: 23,976 windows per frame, 32 frames
per call).

It runs in a process of its own (bench.py starts it): the module links the toolkit's CUDA runtime,
which need not be torch's. The reference's correlate is synchronous and takes host arrays (its copies
are inside the timed calls), so its figure compares with the b200 path's e2e number.

usage: python oracle/ref_cuda_bench.py [--workload hd|stream] [--frames 64]    (prints one JSON line)
"""

import argparse
import importlib.machinery
import importlib.util
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from slipcam_b200 import synth   # noqa: E402
from slipcam_b200.framecor import window_grid   # noqa: E402


def module():
    d = os.path.join(HERE, '_ref', 'cuda')
    names = [f for f in os.listdir(d) if f.startswith('_framecor') and f.endswith('.so')] if os.path.isdir(d) else []
    if not names:
        return None
    path = os.path.join(d, names[0])
    loader = importlib.machinery.ExtensionFileLoader('_framecor', path)
    spec = importlib.util.spec_from_file_location('_framecor', path, loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def main():
    p = argparse.ArgumentParser()
    p.add_argument('--workload', default='hd', choices=['hd', 'stream'])
    p.add_argument('--frames', type=int, default=None, help='frames timed (default 64 at 720p, 64 at 1080p)')
    args = p.parse_args()
    mod = module()
    if mod is None:
        print(json.dumps({'unavailable': 'the reference CUDA backend was not built (make -C oracle ref_cuda)'}))
        return
    if not mod.has_cuda():
        print(json.dumps({'unavailable': 'no GPU'}))
        return
    if args.workload == 'hd':
        H, W, WIN, SEARCH, SKIP, args.batch = 720, 1280, 64, 48, 16, 16
    else:
        H, W, WIN, SEARCH, SKIP, args.batch = 1080, 1920, 64, 64, 8, 32
    frames_timed = args.frames or 64
    down, across = window_grid(H, W, WIN, SEARCH, SKIP)
    nwin = len(down) * len(across)
    n = frames_timed + args.batch   # one call of warm-up
    make = synth.hd if args.workload == 'hd' else synth.stream
    frames, motion, step, gross = make(n=300 if args.workload == 'hd' else 1000, count=n + 1)
    runs = {}
    # the reference's default batch (4096 pairs: one frame per group at 2450 windows, part of one at
    # 23,976), then batches of whole frames up to a call (16 frames at 720p; 2 at 1080p, where the
    # reference's per-batch buffers take 7 GB each)
    whole = min(args.batch, max(1, 48000 // nwin))
    for label, pairs in (('default_batch_4096', 4096), (f'batch_of_{whole}_frames', whole * nwin)):
        cor = mod.Correlator(H, W, list(down), list(across), window=WIN, search=SEARCH, backend='cuda', batch=pairs)
        t = time.perf_counter()
        cor.set_reference(frames[0])
        ref_s = time.perf_counter() - t
        cor.correlate(frames[1:1 + args.batch], gross=gross[1:1 + args.batch])   # warm-up: plans, first launches
        t = time.perf_counter()
        done = 0
        for s in range(1 + args.batch, n + 1 - args.batch + 1, args.batch):
            r = cor.correlate(frames[s:s + args.batch], gross=gross[s:s + args.batch])
            done += args.batch
        dt = time.perf_counter() - t
        runs[label] = {'value': done * nwin / dt, 'ms_per_frame': dt * 1e3 / done, 'set_reference_s': ref_s,
                       'valid_fraction': float(np.isfinite(r['offsets'][..., 0]).mean())}
        del cor
    best = max(runs.values(), key=lambda v: v['value'])
    print(json.dumps({
        'impl': 'reference CUDA backend (cuFFT), sm_100a', 'value': best['value'], 'unit': 'windows/s',
        'workload': args.workload, 'windows_per_frame': nwin, 'frames': done, 'frames_per_call': args.batch,
        'runs': runs,
        'path': 'Correlator(backend="cuda").correlate on host arrays (its H2D / D2H copies and sync inside)',
    }))


if __name__ == '__main__':
    main()
