"""
Dense offsets of the frames of a video relative to a reference frame, streamed through the b200
backend: the driver of python/slipcam/track_offsets.py (track, boxes_mask, main; the same arguments,
the same .npz keys) on the b200 Correlator.

The frames are read from the (memory-mapped) array in chunks into two page-locked buffers by a
reader thread, so the disk, the host-to-device copies and the correlation overlap: while chunk k is
correlated from one buffer, chunk k + 1 is read into the other. Each chunk goes through the
Correlator's host entry point, which pipelines its own launch groups over two streams.

usage:
  python -m slipcam_b200.track run/frames.npy --ref 285 --first 140 --out run/offsets.npz \\
      --mask 870 25 1240 68 --mask 40 650 630 700
"""

import argparse
import threading
import time

import numpy as np

from . import framecor


def boxes_mask(y0, x0, window, boxes):
    """The windows that overlap any of the boxes (x0, y0, x1, y1) (track_offsets.py:27-32)"""
    y0, x0 = np.asarray(y0), np.asarray(x0)
    masked = np.zeros((len(y0), len(x0)), bool)
    for bx0, by0, bx1, by1 in boxes:
        masked |= ((y0[:, None] < by1) & (y0[:, None] + window > by0)
                   & (x0[None, :] < bx1) & (x0[None, :] + window > bx0))
    return masked


class _Reader(threading.Thread):
    """Fills two page-locked buffers with chunks of frames, one chunk ahead of the consumer."""

    def __init__(self, frames, index, chunk, bufs):
        super().__init__(daemon=True)
        self.frames, self.index, self.chunk, self.bufs = frames, index, chunk, bufs
        self.ready = [threading.Semaphore(0), threading.Semaphore(0)]
        self.free = [threading.Semaphore(1), threading.Semaphore(1)]
        self.error = None

    def run(self):
        try:
            for k, k0 in enumerate(range(0, len(self.index), self.chunk)):
                b = k % 2
                self.free[b].acquire()
                sel = self.index[k0:k0 + self.chunk]
                dst = self.bufs[b][:len(sel)]
                if np.array_equal(sel, np.arange(sel[0], sel[0] + len(sel))):   # a run: one slice, no gather
                    np.copyto(dst, self.frames[sel[0]:sel[0] + len(sel)])
                else:
                    np.copyto(dst, self.frames[sel])
                self.ready[b].release()
        except Exception as e:   # handed to the consumer
            self.error = e
            for s in self.ready:
                s.release()


def track(frames, ref, index, masked=None, window=64, skip=16, search=48, cpu=False, chunk=64, form='auto',
          correlator=None):
    """The offsets of the frames index relative to the frame ref, chunk frames per call of the b200
    Correlator; a dict as saved by main (track_offsets.py:35-60). cpu=True is refused: this backend
    has no CPU path. form: the Correlator's arithmetic ('auto' / 'fft32' / 'tc' / 'int8'). correlator: a
    b200 Correlator of this geometry to reuse (its reference is set to frames[ref] here)."""
    if cpu:
        raise ValueError('framecor: the b200 backend has no CPU path (use the reference for cpu=True)')
    import torch
    n, h, w = frames.shape
    y0, x0 = framecor.window_grid(h, w, window, search, skip)
    ny, nx = len(y0), len(x0)
    if masked is None:
        masked = np.zeros((ny, nx), bool)
    cor = correlator or framecor.Correlator(h, w, y0, x0, window=window, search=search, backend='b200')
    if cor.shape != (ny, nx) or cor.window != window or cor.search != search:
        raise ValueError('framecor: the correlator does not match the geometry')
    if form != 'auto':
        cor.set_form(form)
    index = np.asarray(index)
    out = {key: np.empty((len(index), ny, nx) + tail, np.float32)
           for key, tail in (('offsets', (2,)), ('snr', ()), ('cov', (3,)), ('peak', ()))}
    tic = time.perf_counter()
    cor.set_reference(np.ascontiguousarray(frames[ref]))
    if len(index):
        bufs = [torch.empty((min(chunk, len(index)), h, w), dtype=torch.uint8, pin_memory=True).numpy() for _ in range(2)]
        reader = _Reader(frames, index, chunk, bufs)
        reader.start()
        for k, k0 in enumerate(range(0, len(index), chunk)):
            b = k % 2
            reader.ready[b].acquire()
            if reader.error is not None:
                raise reader.error
            m = len(index[k0:k0 + chunk])
            r = cor.correlate(bufs[b][:m])
            reader.free[b].release()
            for key in out:
                out[key][k0:k0 + m] = r[key]
        reader.join()
    elapsed = time.perf_counter() - tic
    per = elapsed / max(len(index), 1) * 1e3
    print(f'tracked {len(index)} frame(s), {ny * nx} windows each ({ny} rows x {nx} columns): {elapsed:.1f} s, '
          f'{per:.1f} ms a frame on the {cor.backend} backend; {int(masked.sum())} window(s) under text boxes')
    return dict(index=index, ref=ref, masked=masked, yc=y0 + window / 2, xc=x0 + window / 2, window=window,
                skip=skip, search=search, engine='framecor', **out)


def main(argv=None):
    parser = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    parser.add_argument('frames', help='video as a uint8 .npy array shaped (count, rows, columns)')
    parser.add_argument('--ref', type=int, required=True, help='index of the frame every other frame is matched to')
    parser.add_argument('--first', type=int, default=0, help='index of the first tracked frame [%(default)s]')
    parser.add_argument('--last', type=int, help='index of the last tracked frame, inclusive [end of the video]')
    parser.add_argument('--window', type=int, default=64, help='side of a square correlation window in px [%(default)s]')
    parser.add_argument('--skip', type=int, default=16, help='step between neighbouring window origins in px [%(default)s]')
    parser.add_argument('--search', type=int, default=48, help='largest offset tried in each direction, px [%(default)s]')
    parser.add_argument('--mask', type=int, nargs=4, action='append', default=[], metavar=('X0', 'Y0', 'X1', 'Y1'),
                        help='pixel box of an overlay (e.g. a timestamp); windows touching it are flagged. May repeat')
    parser.add_argument('--cpu', action='store_true', help='not available here: this backend runs on the GPU only')
    parser.add_argument('--chunk', type=int, default=64, help='frames handed to one correlate call [%(default)s]')
    parser.add_argument('--form', default='auto', choices=['auto', 'fft32', 'tc', 'int8'],
                        help='correlation arithmetic: auto picks per geometry [%(default)s]')
    parser.add_argument('--out', required=True, help='where to write the results (.npz)')
    args = parser.parse_args(argv)

    frames = np.load(args.frames, mmap_mode='r')
    n, h, w = frames.shape
    last = n - 1 if args.last is None else args.last
    y0, x0 = framecor.window_grid(h, w, args.window, args.search, args.skip)
    masked = boxes_mask(y0, x0, args.window, args.mask)
    result = track(frames, args.ref, np.arange(args.first, last + 1), masked=masked, window=args.window,
                   skip=args.skip, search=args.search, cpu=args.cpu, chunk=args.chunk, form=args.form)
    np.savez(args.out, **result)
    print(f'wrote {args.out}')


if __name__ == '__main__':
    main()
