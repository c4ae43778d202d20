"""
Coarse similarity tracking of the frames of a video on a reference frame, on the b200 backend:
stabilize.coarse_track (python/slipcam/stabilize.py:54-96) with its ncc_peak (:22-44) and the robust
fit slip_series.fit_camera (python/slipcam/slip_series.py:49-72); same arguments, same results.

A grid of large windows of the reference frame (away from the burned-in text, not flat) is tracked in
each frame around the positions predicted by the previous frame's transform. Per frame, three
stream-ordered steps on the GPU and no host round trip:

* the correlation of the grid's templates (FP32 FFT correlation, normalized surfaces), each
  window's search window placed by the gross offsets on the device;
* the peak of each surface, refined by a parabola per axis;
* the robust similarity fit of the frame in float64, in one CTA, which writes the frame's transform
  and the next frame's gross offsets.

The frame loop runs in the library (b200_coarse_track_device): per group of frames the tables in one
batch, then three launches per frame.

Frames in host memory are copied from the caller's array on a side stream while the previous chunk
is tracked; CUDA tensors are read in place.

The resampling half of the module, warp and stabilize (stabilize.py:99-124), runs on the GPU too
(csrc/warp.cu): the text blanked with scipy's box means, the frames warped with map_coordinates'
bilinear rule, the fill numpy's float32 mean, each step in the reference's arithmetic.
"""

import ctypes

import numpy as np

from . import _lib, _stage, framecor


def apply(params, x, y):
    """The positions of the points (x, y), relative to the image center, under the similarity
    transform params = (p, q, a, s): x' = x + p - a y + s x, y' = y + q + a x + s y
    (stabilize.py:47-51)"""
    p, q, a, s = params
    return x + p - a * y + s * x, y + q + a * x + s * y


def _check(rc):
    if rc != _lib.OK:
        raise (ValueError if rc == _lib.EINVAL else RuntimeError)(f'framecor: stabilize step failed ({rc})')


def ncc_peaks(surfaces):
    """The peak of each normalized surface (a float32 CUDA tensor ... x M x M) as ncc_peak gives it:
    (dy, dx) relative to the surface centre, refined by a parabola per axis, and the value; a float64
    CUDA tensor ... x 3."""
    import torch
    s = surfaces.to(torch.float32).contiguous()
    M = s.shape[-1]
    if s.dim() < 2 or s.shape[-2] != M:
        raise ValueError('framecor: the surfaces must be ... x M x M')
    n = s.numel() // (M * M) if M else 0
    out = torch.empty(tuple(s.shape[:-2]) + (3,), dtype=torch.float64, device=s.device)
    _check(_lib.lib().b200_ncc_peaks_device(s.data_ptr(), n, M, out.data_ptr(),
                                            torch.cuda.current_stream(s.device).cuda_stream))
    return out


def template_grid(h, w, window, step, search):
    """The centres of the rows and columns of windows of coarse_track (stabilize.py:61-63)"""
    half = window // 2
    return np.arange(search + half, h - search - half, step), np.arange(search + half, w - search - half, step)


def _keep(ref, text, yc, xc, half):
    """The windows without text and not flat (the standard deviation of the reference window above
    2), ny x nx (stabilize.py:65-67)"""
    refimg = np.asarray(ref).astype(np.float64)
    text = np.asarray(text, bool)
    keep = np.zeros((len(yc), len(xc)), bool)
    for i, y in enumerate(yc):
        for j, x in enumerate(xc):
            keep[i, j] = (not text[y - half:y + half, x - half:x + half].any()
                          and refimg[y - half:y + half, x - half:x + half].std() > 2)
    return keep


def _runs(order, chunk):
    """order in pieces of at most chunk frames"""
    return [order[k:k + chunk] for k in range(0, len(order), chunk)]


class CoarseTracker:
    """
    The templates of coarse_track, prepared once: the grid of window x window templates of the
    reference frame ref_frame (height x width uint8) centred search + window // 2 pixels or more inside
    it, step apart, those without text (text: height x width bool) and not flat in use, their spectra
    resident on the GPU. run() tracks a video's frames with them (stabilize.py:54-96).
    """

    def __init__(self, ref_frame, text, window=96, step=96, search=32, min_peak=0.5, device=None):
        import torch
        if window % 2 or window < 2:
            raise ValueError('framecor: coarse_track needs an even window of at least 2 pixels')
        ref_frame = ref_frame.cpu().numpy() if isinstance(ref_frame, torch.Tensor) else np.asarray(ref_frame)
        text = text.cpu().numpy() if isinstance(text, torch.Tensor) else text
        self.height, self.width = h, w = ref_frame.shape
        self.window, self.search, self.min_peak = window, search, float(min_peak)
        half = window // 2
        self.yc, self.xc = template_grid(h, w, window, step, search)
        keep = _keep(ref_frame, text, self.yc, self.xc, half)
        self.count = int(keep.sum())
        self.nwin = keep.size
        self.device = torch.device('cuda', torch.cuda.current_device()) if device is None else torch.device(device)
        self._cor = None
        if self.nwin == 0:   # no window fits the frame
            return
        if self.nwin > _lib.COARSE_MAX_WINDOWS:
            raise ValueError(f'framecor: coarse_track handles up to {_lib.COARSE_MAX_WINDOWS} windows, not {self.nwin}')
        dev = self.device
        self._cor = framecor.Correlator(h, w, self.yc - half, self.xc - half, window=window, search=search,
                                        backend='b200', device=dev.index or 0)
        with torch.cuda.device(dev):
            self._cor.set_reference(torch.as_tensor(np.ascontiguousarray(ref_frame, np.uint8)).to(dev))
            self._keep = torch.as_tensor(keep.astype(np.uint8).ravel()).to(dev)
            self._gross = torch.zeros((self.nwin, 2), dtype=torch.int32, device=dev)
            self._prev = torch.zeros(4, dtype=torch.float64, device=dev)

    def run(self, frames, ref, start=0, chunk=64):
        """(params, used, count) of coarse_track for the frames (n x height x width uint8, a numpy array
        or a CUDA tensor) around the reference frame ref: forward from ref, then backward to start.
        chunk: frames per call of the library (and per host-to-device copy)."""
        import torch
        n, h, w = frames.shape
        if (h, w) != (self.height, self.width):
            raise ValueError('framecor: the frames and the reference frame differ in size')
        if not 0 <= ref < n:
            raise IndexError('framecor: the reference frame is not in the video')
        params = np.full((n, 4), np.nan)
        used = np.zeros(n, int)
        passes = [list(range(ref + 1, n)), list(range(ref - 1, start - 1, -1))]
        order = passes[0] + passes[1]
        params[ref], used[ref] = 0, self.count
        if self._cor is None:   # no window: no fit anywhere, the transforms stay zero
            params[order] = 0
            return params, used, self.count
        dev = self.device
        with torch.cuda.device(dev):
            out = torch.full((len(order), 4), float('nan'), dtype=torch.float64, device=dev)   # in tracking order
            nused = torch.zeros(len(order), dtype=torch.int32, device=dev)
            stream = torch.cuda.current_stream(dev)

            def track(ptr, m, at, reset):
                """m frames at ptr (in tracking order), outputs from row `at` of the order"""
                _lib.raise_for(_lib.lib().b200_coarse_track_device(
                    self._cor._h, ptr, m, w, self._keep.data_ptr(), ctypes.c_double(self.min_peak), int(reset),
                    self._gross.data_ptr(), self._prev.data_ptr(), out[at:].data_ptr(), nused[at:].data_ptr(),
                    stream.cuda_stream), self._cor._h)

            at = 0
            if isinstance(frames, torch.Tensor) and frames.is_cuda:
                f = frames.to(torch.uint8).contiguous()
                for frames_in_order in passes:
                    for c, run in enumerate(_runs(frames_in_order, chunk)):
                        if run[0] < run[-1] or len(run) == 1:   # forward: the frames as they lie
                            track(f[run[0]].data_ptr(), len(run), at, c == 0)
                        else:                                    # backward: a reversed copy of the chunk
                            rev = f[run[-1]:run[0] + 1].flip(0).contiguous()
                            track(rev.data_ptr(), len(run), at, c == 0)
                        at += len(run)
            elif order:
                # each chunk staged through pinned memory on a side stream (a backward chunk reversed
                # on the device), the copy of chunk k + 1 overlapping the tracking of chunk k; two
                # device buffers, each reused once its chunk is tracked
                C = min(chunk, len(order))
                devb = [torch.empty((C, h, w), dtype=torch.uint8, device=dev) for _ in range(2)]
                rev = torch.empty((C, h, w), dtype=torch.uint8, device=dev)
                up = _stage.Uploader((h, w), C, dev)
                done = [None, None]
                b = 0
                for frames_in_order in passes:
                    for c, run in enumerate(_runs(frames_in_order, C)):
                        lo, hi, m = min(run[0], run[-1]), max(run[0], run[-1]) + 1, len(run)
                        if run[0] <= run[-1]:
                            ready = up.put(frames[lo:hi], devb[b][:m], after=done[b])
                        else:
                            up.put(frames[lo:hi], rev[:m])
                            with torch.cuda.stream(up.stream):
                                if done[b] is not None:
                                    up.stream.wait_event(done[b])   # the chunk before last is tracked
                                devb[b][:m].copy_(rev[:m].flip(0))
                                ready = up.stream.record_event()
                        stream.wait_event(ready)
                        track(devb[b].data_ptr(), m, at, c == 0)
                        done[b] = stream.record_event()
                        at += m
                        b ^= 1
            if order:
                params[order] = out.cpu().numpy()
                used[order] = nused.cpu().numpy()
        return params, used, self.count


def coarse_track(frames, ref, text, window=96, step=96, search=32, min_peak=0.5, start=0, *, chunk=64):
    """The similarity transform of each frame relative to the frame ref (frames x 4: p, q, a, s about
    the image center), the number of windows of each frame's fit, and the number of windows of the
    grid in use (stabilize.py:54-96). frames: n x height x width uint8, a numpy array (memory-mapped
    or not) or a CUDA tensor; text: the burned-in text mask (height x width bool). The frames after
    ref are tracked forward from it, then those from ref - 1 down to start backward; each frame is
    predicted from the previous one's transform (zero at the start of each pass). A frame without a
    fit (fewer than 4 windows) keeps the previous transform and counts 0 windows; the frames before
    start stay NaN.

    chunk: frames per call of the library (and per host-to-device copy). The correlation is the FP32
    form. The window must be even (the reference's template is 2 (window // 2) pixels wide)."""
    import torch
    if window % 2 or window < 2:
        raise ValueError('framecor: coarse_track needs an even window of at least 2 pixels')
    if not 0 <= ref < len(frames):
        raise IndexError('framecor: the reference frame is not in the video')
    dev = frames.device if isinstance(frames, torch.Tensor) and frames.is_cuda else None
    tracker = CoarseTracker(frames[ref], text, window=window, step=step, search=search, min_peak=min_peak, device=dev)
    return tracker.run(frames, ref, start=start, chunk=chunk)


def _stab_check(rc, ctx):
    if rc != _lib.OK:
        msg = _lib.lib().b200_stab_last_error(ctx).decode() if ctx else ''
        raise (ValueError if rc == _lib.EINVAL else RuntimeError)(msg or f'framecor: stabilize failed ({rc})')


def warp(frame, params, fill=None):
    """The frame resampled onto the reference (stabilize.py:99-106): the value at (x, y) of the
    reference is that of the frame at the transformed position (bilinear); outside the frame, fill.
    The default fill is the frame's mean: numpy's for a numpy frame (the reference's value); for a
    CUDA tensor its float64 mean, which can differ from numpy's float32 mean in the last bits.
    stabilize() computes numpy's float32 mean on the GPU itself. frame: height x width, a numpy
    array or a CUDA tensor; returns float32 of the same kind."""
    import torch
    on_device = isinstance(frame, torch.Tensor) and frame.is_cuda
    if fill is None:
        fill = frame.double().mean().item() if on_device else np.asarray(frame).mean()
    dev = frame.device if on_device else torch.device('cuda', torch.cuda.current_device())
    f = (frame if on_device else torch.as_tensor(np.ascontiguousarray(frame, np.float32))).to(dev, torch.float32).contiguous()
    if f.dim() != 2:
        raise ValueError('framecor: the frame must be height x width')
    h, w = f.shape
    p = torch.as_tensor(np.asarray(params, np.float64).reshape(4)).to(dev)
    out = torch.empty((h, w), dtype=torch.float32, device=dev)
    with torch.cuda.device(dev):
        _check(_lib.lib().b200_warp_f32_device(f.data_ptr(), h, w, p.data_ptr(), ctypes.c_float(float(np.float32(fill))),
                                               out.data_ptr(), torch.cuda.current_stream(dev).cuda_stream))
    return out if on_device else out.cpu().numpy()


class Stabilizer:
    """
    stabilize's context for one text mask (height x width bool; numpy or torch): the mask, its box
    mean over size x size pixels and the summation plans, on the GPU. run(frames, params) warps
    frames onto the reference (stabilize.py:109-124).
    """

    def __init__(self, text, size=31, device=None):
        import torch
        text = text.cpu().numpy() if isinstance(text, torch.Tensor) else np.asarray(text)
        if text.ndim != 2:
            raise ValueError('framecor: the text mask must be height x width')
        self.height, self.width = text.shape
        self.device = torch.device('cuda', torch.cuda.current_device()) if device is None else torch.device(device)
        t = np.ascontiguousarray(text.astype(bool), np.uint8)
        ctx = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            rc = _lib.lib().b200_stab_create(self.height, self.width, t.ctypes.data, int(size), self.device.index or 0,
                                             ctypes.byref(ctx))
        _stab_check(rc, None)
        self._ctx = ctx

    def __del__(self):
        ctx = getattr(self, '_ctx', None)
        self._ctx = None
        if ctx and _lib is not None and _lib._lib is not None:
            _lib._lib.b200_stab_destroy(ctx)

    def run(self, frames, params, chunk=16):
        """(frames warped onto the reference, uint8, with their text blanked; the union of the warped
        text masks, bool) for frames (n x height x width uint8, numpy or CUDA tensor) and params
        (n x 4: p, q, a, s). Numpy in, numpy out; a CUDA tensor in, CUDA tensors out. chunk: frames
        per host-to-device copy."""
        import torch
        n, h, w = frames.shape
        if (h, w) != (self.height, self.width):
            raise ValueError('framecor: the frames and the text mask differ in size')
        params = params.cpu().numpy() if isinstance(params, torch.Tensor) else np.asarray(params)
        if params.shape != (n, 4):
            raise ValueError('framecor: params must be frames x 4')
        dev = self.device
        on_device = isinstance(frames, torch.Tensor) and frames.is_cuda
        with torch.cuda.device(dev):
            stream = torch.cuda.current_stream(dev)
            p = torch.as_tensor(np.ascontiguousarray(params, np.float64)).to(dev)
            union = torch.zeros((h, w), dtype=torch.uint8, device=dev)
            lib = _lib.lib()

            def run(src, m, k0, dst):
                _stab_check(lib.b200_stab_frames_device(self._ctx, src.data_ptr(), m, w, p[k0:].data_ptr(),
                                                        dst.data_ptr(), union.data_ptr(), stream.cuda_stream), self._ctx)

            if on_device:
                f = frames.to(dev, torch.uint8).contiguous()
                out = torch.empty((n, h, w), dtype=torch.uint8, device=dev)
                if n:
                    run(f, n, 0, out)
                return out, union.bool()
            # two sets of device buffers; chunk k + 1 is staged in through pinned memory (on a side
            # stream) and warped while chunk k is staged out into the result (on another)
            out = np.empty((n, h, w), np.uint8)
            C = max(1, min(chunk, n))
            dev_in = [torch.empty((C, h, w), dtype=torch.uint8, device=dev) for _ in range(2)]
            dev_out = [torch.empty((C, h, w), dtype=torch.uint8, device=dev) for _ in range(2)]
            up, down = _stage.Uploader((h, w), C, dev), _stage.Downloader((h, w), C, dev)
            read_in, read_out = [None, None], [None, None]
            for c, k0 in enumerate(range(0, n, C)):
                b, m = c % 2, min(C, n - k0)
                stream.wait_event(up.put(frames[k0:k0 + m], dev_in[b][:m], after=read_in[b]))
                if read_out[b] is not None:
                    stream.wait_event(read_out[b])   # chunk c - 2 is out of dev_out[b]
                run(dev_in[b], m, k0, dev_out[b])
                read_in[b] = stream.record_event()
                read_out[b] = down.get(dev_out[b][:m], out[k0:k0 + m], after=read_in[b])
            down.flush()
            return out, union.cpu().numpy().astype(bool)


def stabilize(frames, params, text, *, chunk=16):
    """The frames warped onto the reference (uint8), with their text blanked (the local mean), and the
    union of the warped text masks (stabilize.py:109-124). frames: n x height x width uint8 (numpy or
    CUDA tensor); params: n x 4 (coarse_track's transforms); text: height x width bool."""
    import torch
    dev = frames.device if isinstance(frames, torch.Tensor) and frames.is_cuda else None
    return Stabilizer(text, device=dev).run(frames, params, chunk=chunk)
