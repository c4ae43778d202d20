"""
framecor on a B200: dense normalized cross-correlation of video frames with a reference frame.

The same Python API as slipcam's framecor (python/slipcam/framecor/__init__.py and the pybind11
module of cxx/bindings.cpp), with the backend 'b200':

  grid = framecor.window_grid(720, 1280, window=64, search=48, skip=16)
  cor = framecor.Correlator(720, 1280, *grid, window=64, search=48, backend='b200')
  cor.set_reference(frames[ref])
  result = cor.correlate(frames[first:last])     # offsets, peak, snr, cov

The compute runs in libslipcam_b200.so (hand-written sm_100a CUDA) through its C ABI; there is no
CPU path. Inputs may be numpy arrays (outputs are numpy, the reference's behaviour) or CUDA torch
tensors (uint8 frames already on the device; outputs are torch tensors on that device, computed
on the current stream without a host synchronization).
"""

import ctypes

import numpy as np

from . import _lib

__version__ = '0.1.0'
__all__ = ['Correlator', 'has_cuda', 'window_grid', '__version__']


def window_grid(height, width, window, search, skip, margin=0):
    """
    The first pixels (down, across) of the grid of windows whose search windows are in the frame:
    from margin + search, (size - 2 (margin + search) - window) // skip windows in each direction
    (python/slipcam/framecor/__init__.py:18-32); a ValueError if no window fits
    """
    axes = []
    for direction, size in (('down', height), ('across', width)):
        first = margin + search
        count = (size - margin - search - first - window) // skip
        if count <= 0:
            raise ValueError(f'window_grid: no window fits {direction}: frame size {size}, window {window}, '
                             f'search range {search}, margin {margin}')
        axes.append(first + skip * np.arange(count))
    return tuple(axes)


def has_cuda():
    """Whether the b200 backend can run: its library is built and a B200 is present."""
    return _lib.loaded() and bool(_lib.lib().b200_has_device())


def _is_torch(x):
    return type(x).__module__.startswith('torch')


def _u8(a):
    """numpy uint8, C-contiguous (the reference's forcecast, bindings.cpp:21)."""
    return np.ascontiguousarray(np.asarray(a).astype(np.uint8, copy=False))


class Correlator:
    """
    The correlator of 8-bit frames with a reference frame, on a grid of square windows

    height, width: the size of the frames
    down, across: the first pixels of the rows and of the columns of windows
    window: the size of the windows; search: the half search range, pixels
    backend: 'b200' or 'auto' (the b200 backend; there is no other here)
    batch: a hint (the reference's FFT batch); stat_size: the SNR window
    device: the GPU; threads: accepted for compatibility, unused
    """

    def __init__(self, height, width, down, across, *, window=64, search=48, backend='auto', batch=4096,
                 stat_size=21, device=0, threads=0):
        self._h = None
        down = np.ascontiguousarray(np.asarray(down), np.int32)
        across = np.ascontiguousarray(np.asarray(across), np.int32)
        if down.ndim != 1 or across.ndim != 1:
            raise TypeError('framecor: down and across must be sequences of ints')
        self._down, self._across = down, across
        self._p = _lib.Params(int(height), int(width), int(window), int(search), int(stat_size), int(batch),
                              down.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(down),
                              across.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(across))
        if backend not in ('auto', 'b200'):
            self._check_params()
            raise ValueError(f'framecor: the backend must be auto or b200, not {backend}')
        h = ctypes.c_void_p()
        rc = _lib.lib().b200_create(ctypes.byref(self._p), int(device), ctypes.byref(h))
        _lib.raise_for(rc, None)
        self._h = h
        self._height, self._width = int(height), int(width)
        self._window, self._search = int(window), int(search)
        self._ny, self._nx = len(down), len(across)
        self._ready = False

    def _check_params(self):
        # the parameter checks come first in the reference (bindings.cpp:37 before :38-44); a
        # create with device -1 runs them without touching a GPU
        h = ctypes.c_void_p()
        rc = _lib.lib().b200_create(ctypes.byref(self._p), -1, ctypes.byref(h))
        if rc == _lib.EINVAL:
            _lib.raise_for(rc, None)

    def __del__(self):
        h = getattr(self, '_h', None)
        self._h = None
        if h and _lib is not None and _lib._lib is not None:
            _lib._lib.b200_destroy(h)

    @property
    def backend(self):
        return 'b200'

    @property
    def shape(self):
        """the number of windows (down, across)"""
        return (self._ny, self._nx)

    @property
    def window(self):
        return self._window

    @property
    def search(self):
        return self._search

    def set_form(self, form):
        """The arithmetic of the transforms: 'fft32' (FP32 FFTs on the CUDA cores), 'tc' (DFT-matrix
        GEMMs on the tensor cores, FP16 operands, FP32 accumulation), 'int8' (the correlation summed
        directly on the tensor cores in exact integers, then normalized) or 'auto'."""
        code = {'auto': _lib.FORM_AUTO, 'fft32': _lib.FORM_FFT32, 'tc': _lib.FORM_TC,
                'int8': _lib.FORM_I8}.get(form)
        if code is None:
            raise ValueError(f'framecor: unknown form {form}')
        _lib.raise_for(_lib.lib().b200_set_form(self._h, code), self._h)

    def check(self, stream=None):
        """After device-path calls (CUDA tensors, no host synchronization): wait for them and raise
        RuntimeError if a bounded wait inside a tensor-core kernel gave up since the last check (their
        outputs are not valid). The host-array path checks by itself."""
        import torch
        st = ctypes.c_int()
        s = (stream if stream is not None else torch.cuda.current_stream()).cuda_stream
        _lib.raise_for(_lib.lib().b200_status(self._h, s, ctypes.byref(st)), self._h)
        if st.value:
            raise RuntimeError('framecor: a tensor-core completion wait gave up; the outputs are not valid')

    def info(self):
        """(ny, nx, fft_size, kernel launches so far)"""
        ny, nx, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        launches = ctypes.c_uint64()
        _lib.lib().b200_info(self._h, ctypes.byref(ny), ctypes.byref(nx), ctypes.byref(n), ctypes.byref(launches))
        return ny.value, nx.value, n.value, launches.value

    def profile(self, enable=True):
        """Bracket every correlation-kernel launch with CUDA events (see profile_read)."""
        _lib.raise_for(_lib.lib().b200_profile(self._h, int(bool(enable))), self._h)

    def profile_read(self):
        """(summed correlation-kernel time in ms, its launches, the pairs they processed) since
        the last read."""
        ms, n, pairs = ctypes.c_double(), ctypes.c_uint64(), ctypes.c_uint64()
        _lib.raise_for(_lib.lib().b200_profile_read(self._h, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(pairs)),
                       self._h)
        return ms.value, n.value, pairs.value

    def set_reference(self, frame):
        """Set the reference frame (height x width, uint8)"""
        if _is_torch(frame) and frame.is_cuda:
            import torch
            if frame.dim() != 2 or tuple(frame.shape) != (self._height, self._width):
                raise ValueError('framecor: the reference frame must be height x width')
            f = frame.to(torch.uint8).contiguous()
            stream = torch.cuda.current_stream(f.device).cuda_stream
            rc = _lib.lib().b200_set_reference_device(self._h, f.data_ptr(), self._width, stream)
            _lib.raise_for(rc, self._h)
            torch.cuda.current_stream(f.device).synchronize()
        else:
            f = _u8(frame)
            if f.ndim != 2 or f.shape != (self._height, self._width):
                raise ValueError('framecor: the reference frame must be height x width')
            _lib.raise_for(_lib.lib().b200_set_reference(self._h, f.ctypes.data), self._h)
        self._ready = True

    def _gross(self, gross, n, xp):
        if gross is None:
            return None, _lib.GROSS_NONE
        if xp is np:
            g = np.ascontiguousarray(np.asarray(gross).astype(np.int32, copy=False))
        else:
            g = gross.to(xp.int32).contiguous()
        shape = tuple(g.shape)
        if shape == (n, 2):
            return g, _lib.GROSS_FRAME
        if shape == (n, self._ny, self._nx, 2):
            return g, _lib.GROSS_WINDOW
        raise ValueError('framecor: gross must be frames x 2 or frames x down x across x 2')

    def correlate(self, frames, gross=None, *, surfaces=False):
        """
        Correlate the frames (frames x height x width, uint8) with the reference frame

        gross: integer offsets (down, across) of the search windows, frames x 2 or
        frames x down x across x 2 (default: none)

        Returns a dict of float32 arrays: offsets (frames x down x across x 2: down, across, the
        motion of the frame; NaN if not valid), peak (the normalized correlation), snr, cov (the
        covariance of the offsets: down, across, cross). With surfaces=True (CUDA tensors only)
        also 'surface', the normalized correlation surfaces (frames x down x across x M x M).
        """
        if not self._ready:
            raise RuntimeError('framecor: set_reference first')
        if _is_torch(frames) and frames.is_cuda:
            return self._correlate_device(frames, gross, surfaces)
        if surfaces:
            raise ValueError('framecor: surfaces are returned for CUDA tensor inputs only')
        f = _u8(frames)
        if f.ndim != 3 or f.shape[1] != self._height or f.shape[2] != self._width:
            raise ValueError('framecor: the frames must be frames x height x width')
        n, ny, nx = f.shape[0], self._ny, self._nx
        g, mode = self._gross(gross, n, np)
        out = dict(offsets=np.empty((n, ny, nx, 2), np.float32), peak=np.empty((n, ny, nx), np.float32),
                   snr=np.empty((n, ny, nx), np.float32), cov=np.empty((n, ny, nx, 3), np.float32))
        if n > 0:
            rc = _lib.lib().b200_correlate(self._h, f.ctypes.data, n, None if g is None else g.ctypes.data, mode,
                                           out['offsets'].ctypes.data, out['peak'].ctypes.data,
                                           out['snr'].ctypes.data, out['cov'].ctypes.data)
            _lib.raise_for(rc, self._h)
        return out

    def _correlate_device(self, frames, gross, surfaces):
        import torch
        if frames.dim() != 3 or frames.shape[1] != self._height or frames.shape[2] != self._width:
            raise ValueError('framecor: the frames must be frames x height x width')
        f = frames.to(torch.uint8).contiguous()
        n, ny, nx, dev = f.shape[0], self._ny, self._nx, f.device
        g, mode = self._gross(gross, n, torch)
        if g is not None:
            g = g.to(dev)
        out = dict(offsets=torch.empty((n, ny, nx, 2), dtype=torch.float32, device=dev),
                   peak=torch.empty((n, ny, nx), dtype=torch.float32, device=dev),
                   snr=torch.empty((n, ny, nx), dtype=torch.float32, device=dev),
                   cov=torch.empty((n, ny, nx, 3), dtype=torch.float32, device=dev))
        M = 2 * self._search + 1
        if surfaces:
            out['surface'] = torch.empty((n, ny, nx, M, M), dtype=torch.float32, device=dev)
        if n > 0:
            stream = torch.cuda.current_stream(dev).cuda_stream
            gp = None if g is None else g.data_ptr()
            args = [self._h, f.data_ptr(), n, self._width, gp, mode, out['offsets'].data_ptr(),
                    out['peak'].data_ptr(), out['snr'].data_ptr(), out['cov'].data_ptr()]
            if surfaces:
                rc = _lib.lib().b200_correlate_device_surfaces(*args, out['surface'].data_ptr(), stream)
            else:
                rc = _lib.lib().b200_correlate_device(*args, stream)
            _lib.raise_for(rc, self._h)
        return out


def sat(frames):
    """The summed-area tables of uint8 CUDA frames (n, h, w): (sat uint32 as int64 tensor,
    sat2 int64), each (n, h + 1, w + 1); the first row and column are zero."""
    import torch
    f = frames.to(torch.uint8).contiguous()
    n, h, w = f.shape
    s32 = torch.empty((n, h + 1, w + 1), dtype=torch.int32, device=f.device)
    s64 = torch.empty((n, h + 1, w + 1), dtype=torch.int64, device=f.device)
    stream = torch.cuda.current_stream(f.device).cuda_stream
    rc = _lib.lib().b200_sat_device(f.data_ptr(), n, h, w, w, s32.data_ptr(), s64.data_ptr(), stream)
    if rc != _lib.OK:
        raise ValueError('framecor: sat: invalid arguments')
    return s32.to(torch.int64) & 0xFFFFFFFF, s64


def periodicity(ref, y0, x0, window, search, exclude=5):
    """
    auto_slip.periodicity (python/slipcam/auto_slip.py:105-129) on the b200 backend: the second peak
    of the normalized correlation of each window with its own surroundings in the reference frame
    (1 for a periodic or flat texture, small for a unique one), as a float64 (len(y0), len(x0))
    array. The surfaces are the b200 correlation of the frame with itself (FP32); the peak search
    runs on the GPU. ref: uint8 (height, width), numpy or a CUDA tensor.
    """
    import torch
    f = torch.as_tensor(np.asarray(ref) if not _is_torch(ref) else ref)
    if f.dim() != 2:
        raise ValueError('framecor: the reference frame must be height x width')
    f = f.to(torch.uint8).cuda().contiguous()
    h, w = f.shape
    cor = Correlator(h, w, y0, x0, window=window, search=search, backend='b200')
    cor.set_form('fft32')   # surfaces to the FP32 form's accuracy
    cor.set_reference(f)
    surf = cor.correlate(f[None], surfaces=True)['surface']
    ny, nx = cor.shape
    out = torch.empty(ny * nx, dtype=torch.float32, device=f.device)
    stream = torch.cuda.current_stream(f.device).cuda_stream
    rc = _lib.lib().b200_periodicity_device(cor._h, surf.data_ptr(), int(exclude), out.data_ptr(), stream)
    _lib.raise_for(rc, cor._h)
    return out.view(ny, nx).cpu().numpy().astype(np.float64)


class MultiCorrelator:
    """
    Several window grids (window sizes, search ranges, grids) of one video correlated together:
    one persistent launch over every grid's (window, frame) pairs, the step captured in a CUDA
    graph (b200 backend only; the reference correlates one grid per Correlator).

    grids: a list of dicts with keys down, across, window, search (as for Correlator); up to 4.
    correlate(frames, gross=None) takes uint8 CUDA frames (n x height x width) and, per grid, a
    gross offset array or None, and returns one output dict per grid, as Correlator.correlate.
    tune(frames, gross=None) picks the launch configuration by timing the candidates.
    """

    def __init__(self, height, width, grids, *, stat_size=21, device=0):
        if not 1 <= len(grids) <= 4:
            raise ValueError('framecor: a group holds 1 to 4 grids')
        self._height, self._width = height, width
        self.grids = [Correlator(height, width, g['down'], g['across'], window=g['window'], search=g['search'],
                                 backend='b200', stat_size=stat_size, device=device) for g in grids]
        self._g = None
        hs = (ctypes.c_void_p * len(self.grids))(*[c._h for c in self.grids])
        g = ctypes.c_void_p()
        rc = _lib.lib().b200_group_create(hs, len(self.grids), ctypes.byref(g))
        _lib.raise_for(rc, None, group=True)
        self._g = g

    def __del__(self):
        g = getattr(self, '_g', None)
        self._g = None
        if g is not None and _lib is not None and _lib._lib is not None:
            _lib._lib.b200_group_destroy(g)

    def set_reference(self, frame):
        """The reference frame of every grid."""
        for c in self.grids:
            c.set_reference(frame)

    def _args(self, frames, gross):
        import torch
        if not (_is_torch(frames) and frames.is_cuda):
            raise ValueError('framecor: MultiCorrelator takes CUDA frames')
        if frames.dim() != 3 or frames.shape[1] != self._height or frames.shape[2] != self._width:
            raise ValueError('framecor: the frames must be frames x height x width')
        f = frames.to(torch.uint8).contiguous()
        n, k = f.shape[0], len(self.grids)
        gross = [None] * k if gross is None else list(gross)
        if len(gross) != k:
            raise ValueError('framecor: one gross entry per grid')
        gs, modes, keep = [], [], []
        for c, g in zip(self.grids, gross):
            if g is None:
                gs.append(None)
                modes.append(0)
                continue
            t, mode = c._gross(torch.as_tensor(g), n, torch)
            t = t.to(f.device)
            keep.append(t)
            gs.append(t.data_ptr())
            modes.append(mode)
        gp = (ctypes.c_void_p * k)(*gs)
        mp = (ctypes.c_int * k)(*modes)
        return f, n, gp, mp, keep

    def correlate(self, frames, gross=None):
        import torch
        f, n, gp, mp, keep = self._args(frames, gross)
        outs = []
        for c in self.grids:
            ny, nx = c.shape
            outs.append(dict(offsets=torch.empty((n, ny, nx, 2), dtype=torch.float32, device=f.device),
                             peak=torch.empty((n, ny, nx), dtype=torch.float32, device=f.device),
                             snr=torch.empty((n, ny, nx), dtype=torch.float32, device=f.device),
                             cov=torch.empty((n, ny, nx, 3), dtype=torch.float32, device=f.device)))
        if n:
            k = len(self.grids)
            ptrs = {key: (ctypes.c_void_p * k)(*[o[key].data_ptr() for o in outs]) for key in ('offsets', 'peak', 'snr', 'cov')}
            stream = torch.cuda.current_stream(f.device).cuda_stream
            rc = _lib.lib().b200_group_correlate_device(self._g, f.data_ptr(), n, self._width, gp, mp, ptrs['offsets'],
                                                        ptrs['peak'], ptrs['snr'], ptrs['cov'], stream)
            _lib.raise_for(rc, self._g, group=True)
        del keep
        return outs

    def tune(self, frames, gross=None):
        """Time the launch configurations on these frames and keep the fastest; returns
        (ms per launch, config)."""
        import torch
        f, n, gp, mp, keep = self._args(frames, gross)
        ms = ctypes.c_double()
        stream = torch.cuda.current_stream(f.device).cuda_stream
        rc = _lib.lib().b200_group_tune(self._g, f.data_ptr(), n, self._width, gp, mp, stream, ctypes.byref(ms))
        _lib.raise_for(rc, self._g, group=True)
        del keep
        return ms.value, self.config()

    def config(self):
        """threads per CTA, pairs per work item, costliest grid first, per-grid kernels instead of
        the persistent launch, CUDA graph replay"""
        t, c, f, pg, g = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.raise_for(_lib.lib().b200_group_config(self._g, ctypes.byref(t), ctypes.byref(c), ctypes.byref(f),
                                                   ctypes.byref(pg), ctypes.byref(g)), self._g, group=True)
        return dict(threads=t.value, chunk=c.value, costly_first=bool(f.value), per_grid=bool(pg.value),
                    graph=bool(g.value))

    def set_config(self, threads=256, chunk=1, costly_first=True, per_grid=False, graph=True):
        rc = _lib.lib().b200_group_set_config(self._g, threads, chunk, int(costly_first), int(per_grid), int(graph))
        _lib.raise_for(rc, self._g, group=True)
