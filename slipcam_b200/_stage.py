"""
Host frames to and from the device through pinned staging buffers. A pageable copy goes through the
driver's own staging at about a fifth of the link's rate; here the copy between the caller's array
and pinned memory is split over a pool of up to 8 threads (numpy releases the GIL for it; 16 ran
slower beside the DMA) and the DMA of one buffer overlaps the filling of the next. Used by the
host-memory paths of scans and stabilize.
"""

import os
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np

_POOL = None
_POOL_LOCK = threading.Lock()
_PIECE = 1 << 22   # bytes per task of a split copy


def _pool():
    global _POOL
    with _POOL_LOCK:
        if _POOL is None:
            _POOL = ThreadPoolExecutor(max(1, min(8, os.cpu_count() or 1)), thread_name_prefix="framecor-stage")
        return _POOL


def _pieces(dst, src):
    """the copy of src into dst (same shape) as (dst, src) pairs of about _PIECE bytes: along the
    bytes of both when both are C-contiguous, else along the first axis"""
    if dst.flags.c_contiguous and src.flags.c_contiguous:
        d, s = dst.reshape(-1).view(np.uint8), src.reshape(-1).view(np.uint8)
        return [(d[i:i + _PIECE], s[i:i + _PIECE]) for i in range(0, d.size, _PIECE)]
    per = max(1, _PIECE // max(1, dst[0].nbytes)) if len(dst) else 1
    return [(dst[i:i + per], src[i:i + per]) for i in range(0, len(dst), per)]


def _copy(d, s):
    """one piece: the library's streaming-store copy when both sides are contiguous bytes of the same
    size (it skips reading the destination lines first; ctypes releases the GIL), else np.copyto"""
    if d.flags.c_contiguous and s.flags.c_contiguous and d.nbytes == s.nbytes and d.dtype == s.dtype:
        from . import _lib
        if _lib.lib().b200_host_copy(d.ctypes.data, s.ctypes.data, d.nbytes) == _lib.OK:
            return
    np.copyto(d, s)


def parallel_copy(dst, src):
    """np.copyto(dst, src) split over the staging threads"""
    parts = _pieces(dst, src)
    if len(parts) <= 1:
        _copy(dst, src)
        return
    for f in [_pool().submit(_copy, d, s) for d, s in parts]:
        f.result()


class Uploader:
    """Copies numpy frames (m x h x w uint8, m <= chunk) into device tensors on a copy stream:
    `put(src, dst, after)` fills one of `nbuf` pinned buffers (once the DMA that last read it has
    finished), starts its DMA into dst after the CUDA event `after` (the last reader of dst) and
    returns the event that marks the copy done."""

    def __init__(self, frame_shape, chunk, device, nbuf=3):
        import torch
        self.chunk = chunk
        self.bufs = [torch.empty((chunk, *frame_shape), dtype=torch.uint8, pin_memory=True) for _ in range(nbuf)]
        self.read = [None] * nbuf
        self.stream = torch.cuda.Stream(device)
        self.k = 0

    def put(self, src, dst, after=None):
        import torch
        m = len(src)
        if m > self.chunk:
            raise ValueError('framecor: more frames than the staging buffer holds')
        b = self.k % len(self.bufs)
        self.k += 1
        if self.read[b] is not None:
            self.read[b].synchronize()
        pin = self.bufs[b][:m]
        parallel_copy(pin.numpy(), src)
        with torch.cuda.stream(self.stream):
            if after is not None:
                self.stream.wait_event(after)
            dst.copy_(pin, non_blocking=True)
            ev = self.stream.record_event()
        self.read[b] = ev
        return ev


class Downloader:
    """Copies device frames into numpy arrays: `get(src, dst, after)` waits on a copy stream for the
    event `after` (the kernel that wrote src), DMAs src into a pinned buffer and copies it into dst
    over the staging threads once the DMA is done. `flush()` finishes the copy still pending."""

    def __init__(self, frame_shape, chunk, device, nbuf=2):
        import torch
        self.chunk = chunk
        self.bufs = [torch.empty((chunk, *frame_shape), dtype=torch.uint8, pin_memory=True) for _ in range(nbuf)]
        self.stream = torch.cuda.Stream(device)
        self.pending = None   # (event, pinned view, destination)
        self.k = 0

    def get(self, src, dst, after):
        import torch
        m = len(src)
        if m > self.chunk:
            raise ValueError('framecor: more frames than the staging buffer holds')
        b = self.k % len(self.bufs)
        self.k += 1
        pin = self.bufs[b][:m]
        with torch.cuda.stream(self.stream):
            self.stream.wait_event(after)
            pin.copy_(src, non_blocking=True)
            ev = self.stream.record_event()
        self.flush()   # the copy before this one (its buffer is the other one)
        self.pending = (ev, pin, dst)
        return ev

    def flush(self):
        if self.pending is not None:
            ev, pin, dst = self.pending
            self.pending = None
            ev.synchronize()
            parallel_copy(dst, pin.numpy())
