"""
The frame scans of auto_slip (python/slipcam/auto_slip.py:56-94) on the b200 backend: the mean
absolute difference of consecutive frames and the burned-in text mask, as CUDA passes over the
uint8 frames (csrc/scans.cuh). Same arguments and results as the reference functions; frames are a
numpy array (memory-mapped or not; copied to the GPU in chunks) or a CUDA tensor.
"""

import numpy as np

from . import _lib, _stage


def _check(rc):
    if rc != _lib.OK:
        raise (ValueError if rc == _lib.EINVAL else RuntimeError)(f'framecor: scan failed ({rc})')


def _device(frames, a, b):
    """frames[a:b] as a contiguous uint8 CUDA tensor"""
    import torch
    if isinstance(frames, torch.Tensor):
        return frames[a:b].to(device='cuda', dtype=torch.uint8).contiguous()
    return torch.as_tensor(np.ascontiguousarray(frames[a:b], np.uint8)).cuda()


def frame_differences(frames, chunk=50):
    """The mean absolute difference of consecutive frames, float32 (n - 1,) (auto_slip.py:56-63)"""
    import torch
    n = len(frames)
    if n < 2:
        return np.empty(0, np.float32)
    h, w = frames.shape[1:]
    out = torch.empty(n - 1, dtype=torch.float32, device='cuda')
    sums = torch.empty(n - 1, dtype=torch.int64, device='cuda')
    stream = torch.cuda.current_stream()
    lib = _lib.lib()

    def scan(f, a, m):
        _check(lib.b200_frame_diff_device(f.data_ptr(), m, h, w, w, out[a:].data_ptr(), sums[a:].data_ptr(),
                                          stream.cuda_stream))
    if isinstance(frames, torch.Tensor):
        for a in range(0, n - 1, chunk):   # chunk + 1 frames: the pairs (a, a + 1) .. (b - 2, b - 1)
            b = min(a + chunk + 1, n)
            scan(_device(frames, a, b), a, b - a)
        return out.cpu().numpy()
    # host frames: staged through pinned memory, the copy of a chunk overlapping the scan of the last
    C = min(chunk, n - 1) + 1
    up = _stage.Uploader((h, w), C, stream.device)
    bufs = [torch.empty((C, h, w), dtype=torch.uint8, device='cuda') for _ in range(2)]
    done = [None, None]
    for i, a in enumerate(range(0, n - 1, chunk)):
        b, k = min(a + chunk + 1, n), i % 2
        stream.wait_event(up.put(frames[a:b], bufs[k][:b - a], after=done[k]))
        scan(bufs[k], a, b - a)
        done[k] = stream.record_event()
    return out.cpu().numpy()


def percentile(x, q):
    """numpy.percentile(x, q) (method 'linear') of a float32 CUDA tensor, as numpy computes it for
    float32 data; a float32 scalar. The selection runs on the device (csrc/scans.cuh)."""
    import torch
    if not (isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == torch.float32):
        raise TypeError('framecor: percentile takes a float32 CUDA tensor')
    v = x.contiguous()
    out = torch.empty(1, dtype=torch.float32, device=v.device)
    scratch = torch.empty(_lib.PERCENTILE_SCRATCH, dtype=torch.uint8, device=v.device)
    _check(_lib.lib().b200_percentile_f32_device(v.data_ptr(), v.numel(), float(q), out.data_ptr(), scratch.data_ptr(),
                                                 torch.cuda.current_stream().cuda_stream))
    return np.float32(out.item())


def text_mask(frames, start, nframes=150, chunk=10, edge_percentile=90, max_std=1.5, dilate=4):
    """The pixels of burned-in text, bool (height, width) (auto_slip.py:81-94): strong edges of the
    frame start (above the edge_percentile of its Sobel magnitude) whose values hardly change (the
    median over chunks of the temporal standard deviation below max_std), dilated and with the
    regions they enclose filled."""
    import torch
    n = len(frames)
    h, w = frames.shape[1:]
    starts = list(range(start, min(start + nframes, n) - chunk + 1, chunk))
    if not starts:
        raise ValueError('framecor: no complete chunk of frames for the text mask')
    stream = torch.cuda.current_stream().cuda_stream
    if isinstance(frames, torch.Tensor):
        f = _device(frames, starts[0], starts[-1] + chunk)
    else:   # staged through pinned memory, 32 frames at a time
        f = torch.empty((starts[-1] + chunk - starts[0], h, w), dtype=torch.uint8, device='cuda')
        up = _stage.Uploader((h, w), 32, f.device)
        ev = None
        for k in range(0, len(f), 32):
            ev = up.put(frames[starts[0] + k:starts[0] + min(k + 32, len(f))], f[k:k + 32])
        torch.cuda.current_stream().wait_event(ev)
    sd = torch.empty((h, w), dtype=torch.float32, device='cuda')
    _check(_lib.lib().b200_chunk_std_median_device(f.data_ptr(), len(starts), chunk, h, w, w, sd.data_ptr(), stream))
    ref = f[start - starts[0]:start - starts[0] + 1]
    edge = torch.empty((h, w), dtype=torch.float32, device='cuda')
    _check(_lib.lib().b200_sobel_device(ref.data_ptr(), h, w, w, edge.data_ptr(), stream))
    mask = torch.empty((h, w), dtype=torch.uint8, device='cuda')
    scratch = torch.empty(_lib.lib().b200_text_mask_scratch_bytes(h, w), dtype=torch.uint8, device='cuda')
    _check(_lib.lib().b200_text_mask_device(edge.data_ptr(), sd.data_ptr(), h, w, float(edge_percentile), float(max_std),
                                            int(dilate), mask.data_ptr(), scratch.data_ptr(), scratch.numel(), stream))
    return mask.cpu().numpy().view(bool)   # the kernel writes 0 or 1
