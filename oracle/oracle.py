"""
TEST INFRASTRUCTURE: Python access to the oracle. Imported only by tests/, __graft_entry__.smoke()
and bench.py's CPU leg, as the checker; the product never imports it.

Two oracles:

* ``correlate(...)``: our C restatement of framecor's CPU path (oracle/framecor_oracle.c), in
  the reference's float arithmetic (``mode='ref32'``) or entirely in double (``mode='f64'``),
  with the correlation summed directly (no FFT).
* ``reference_module()``: the reference's own CPU backend and pybind11 module (slipcam
  cxx/cpu.cpp, cxx/common.cpp, cxx/bindings.cpp), compiled unchanged by oracle/Makefile with the
  project's FFTW-API shim (oracle/fftw_shim) standing in for FFTW. Its ``Correlator`` has the
  reference API (bindings.cpp:111-142) with ``backend='cpu'``.

Both are built by ``make -C oracle`` (``build()`` in __graft_entry__.py runs it).
"""

import ctypes
import importlib.machinery
import importlib.util
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'liboracle.so')
REF_DIR = os.path.join(HERE, '_ref')

MODES = {'ref32': 0, 'f64': 1}


class _Params(ctypes.Structure):
    _fields_ = [('height', ctypes.c_int), ('width', ctypes.c_int), ('window', ctypes.c_int),
                ('search', ctypes.c_int), ('stat_size', ctypes.c_int),
                ('down', ctypes.POINTER(ctypes.c_int)), ('ny', ctypes.c_int),
                ('across', ctypes.POINTER(ctypes.c_int)), ('nx', ctypes.c_int)]


_lib = None


def build():
    """Compile the oracle library (and the reference module when its sources are present)."""
    targets = ['oracle']
    if os.path.isdir('/root/reference/cxx'):
        targets += ['ref', 'ref_cuda']
    subprocess.run(['make', '-s', '-C', HERE, *targets], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.orc_correlate.restype = ctypes.c_int
        _lib.orc_correlate.argtypes = [ctypes.POINTER(_Params), ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        _lib.orc_sat.restype = None
        _lib.orc_sat.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                 ctypes.c_void_p]
        _lib.orc_reference_windows.restype = ctypes.c_int
        _lib.orc_reference_windows.argtypes = [ctypes.POINTER(_Params), ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.c_void_p]
    return _lib


def window_grid(height, width, window, search, skip, margin=0):
    """The grid of windows, restated from python/slipcam/framecor/__init__.py:18-32."""
    axes = []
    for size in (height, width):
        first = margin + search
        count = (size - margin - search - first - window) // skip
        if count <= 0:
            raise ValueError('window_grid: no window fits')
        axes.append(first + skip * np.arange(count))
    return tuple(axes)


def _params(height, width, down, across, window, search, stat_size):
    down = np.ascontiguousarray(down, np.int32)
    across = np.ascontiguousarray(across, np.int32)
    p = _Params(height, width, window, search, stat_size,
                down.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(down),
                across.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(across))
    return p, (down, across)


def expand_gross(gross, n, ny, nx):
    """Per-pair gross offsets (n, ny, nx, 2) int32 from (n, 2) or (n, ny, nx, 2), as
    cxx/bindings.cpp:64-80 expands them."""
    if gross is None:
        return None
    g = np.asarray(gross, np.int32)
    if g.shape == (n, 2):
        return np.ascontiguousarray(np.broadcast_to(g[:, None, None, :], (n, ny, nx, 2)))
    if g.shape == (n, ny, nx, 2):
        return np.ascontiguousarray(g)
    raise ValueError('gross must be frames x 2 or frames x down x across x 2')


def sat(frame):
    """The exact int64 summed-area tables (h+1, w+1) of a uint8 frame and of its squares."""
    frame = np.ascontiguousarray(frame, np.uint8)
    h, w = frame.shape
    s = np.empty((h + 1, w + 1), np.int64)
    s2 = np.empty((h + 1, w + 1), np.int64)
    lib().orc_sat(frame.ctypes.data, h, w, s.ctypes.data, s2.ctypes.data)
    return s, s2


def reference_windows(height, width, down, across, window, reference):
    """The zero-mean reference windows (nwin, W, W) float32 and their norms (nwin,) float32."""
    p, keep = _params(height, width, down, across, window, 1, 21)
    ref = np.ascontiguousarray(reference, np.uint8)
    nwin = len(down) * len(across)
    win = np.empty((nwin, window, window), np.float32)
    norms = np.empty(nwin, np.float32)
    lib().orc_reference_windows(ctypes.byref(p), ref.ctypes.data, win.ctypes.data, norms.ctypes.data)
    return win, norms


def correlate(height, width, down, across, reference, frames, gross=None, *, window=64, search=48,
              stat_size=21, mode='f64', surfaces=False, threads=0):
    """The outputs of framecor's correlate for the frames, from the C restatement.

    Returns a dict like the reference's (offsets, peak, snr, cov, float32, shaped
    (n, ny, nx, ...)), plus 'offsets64' (float64) and, if surfaces, 'surface' (n, ny, nx, M, M)
    float64 normalized surfaces.
    """
    frames = np.ascontiguousarray(frames, np.uint8)
    n = frames.shape[0]
    ny, nx = len(down), len(across)
    p, keep = _params(height, width, down, across, window, search, stat_size)
    g = expand_gross(gross, n, ny, nx)
    ref = np.ascontiguousarray(reference, np.uint8)
    M = 2 * search + 1
    out = dict(offsets=np.empty((n, ny, nx, 2), np.float32), peak=np.empty((n, ny, nx), np.float32),
               snr=np.empty((n, ny, nx), np.float32), cov=np.empty((n, ny, nx, 3), np.float32),
               offsets64=np.empty((n, ny, nx, 2), np.float64))
    surf = np.empty((n, ny, nx, M, M), np.float64) if surfaces else None
    rc = lib().orc_correlate(ctypes.byref(p), ref.ctypes.data, frames.ctypes.data, n,
                             None if g is None else g.ctypes.data, MODES[mode],
                             out['offsets'].ctypes.data, out['peak'].ctypes.data,
                             out['snr'].ctypes.data, out['cov'].ctypes.data,
                             out['offsets64'].ctypes.data, None if surf is None else surf.ctypes.data,
                             threads)
    if rc != 0:
        raise ValueError(f'oracle: invalid parameters ({rc})')
    if surfaces:
        out['surface'] = surf
    return out


_ref_module = None


def reference_module():
    """The reference's pybind11 module _framecor (CPU backend, FFT by the shim), from
    oracle/_ref; None if it was not built."""
    global _ref_module
    if _ref_module is None:
        if not os.path.isdir(REF_DIR):
            return None
        names = [f for f in os.listdir(REF_DIR) if f.startswith('_framecor') and f.endswith('.so')]
        if not names:
            return None
        path = os.path.join(REF_DIR, names[0])
        loader = importlib.machinery.ExtensionFileLoader('_framecor', path)
        spec = importlib.util.spec_from_file_location('_framecor', path, loader=loader)
        mod = importlib.util.module_from_spec(spec)
        loader.exec_module(mod)
        sys.modules.setdefault('_oracle_ref_framecor', mod)
        _ref_module = mod
    return _ref_module


def periodicity(ref, y0, x0, window, search, exclude=5):
    """
    TEST INFRASTRUCTURE. The restatement of auto_slip.periodicity (python/slipcam/auto_slip.py:105-129):
    for each window of the uint8 reference frame, its normalized correlation with its own
    surroundings (the FP64 direct oracle's surface, the search window around the window itself),
    the 5 x 5 local maxima of that surface with reflecting borders (scipy.ndimage.maximum_filter's
    default), without those in the (2 exclude + 1)^2 box around zero shift (the same slice as the
    reference, negative starts included), and the largest of them; 1 for a flat window (norm below
    1e-6), 0 if no peak is left.
    """
    ref = np.ascontiguousarray(ref, np.uint8)
    h, w = ref.shape
    y0, x0 = np.asarray(y0), np.asarray(x0)
    o = correlate(h, w, y0, x0, ref, ref[None], None, window=window, search=search, mode='f64', surfaces=True)
    _, norms = reference_windows(h, w, y0, x0, window, ref)
    norms = np.asarray(norms).reshape(len(y0), len(x0))
    out = np.ones((len(y0), len(x0)))
    c = search
    for i in range(len(y0)):
        for j in range(len(x0)):
            if norms[i, j] < 1e-6:
                continue
            s = o['surface'][0, i, j].astype(np.float64)
            local = np.lib.stride_tricks.sliding_window_view(np.pad(s, 2, mode='symmetric'), (5, 5)).max(axis=(-2, -1))
            peaks = s == local
            peaks[c - exclude:c + exclude + 1, c - exclude:c + exclude + 1] = False
            out[i, j] = s[peaks].max() if peaks.any() else 0.0
    return out


def frame_differences(frames, chunk=50):
    """
    TEST INFRASTRUCTURE. The restatement of auto_slip.frame_differences (auto_slip.py:56-63): the
    mean absolute difference of consecutive uint8 frames, from exact integer sums (float32 result).
    """
    f = np.asarray(frames)
    out = np.empty(len(f) - 1, np.float32)
    for k in range(len(f) - 1):
        s = np.abs(f[k + 1].astype(np.int64) - f[k].astype(np.int64)).sum()
        out[k] = np.float32(s / f[k].size)
    return out


def _sobel_magnitude(img):
    """hypot of the two Sobel derivatives of a float32 image, borders reflected (half-sample)"""
    p = np.pad(img.astype(np.float64), 1, mode='symmetric')
    rows = lambda d: p[1 + d:p.shape[0] - 1 + d]
    cols = lambda a, d: a[:, 1 + d:a.shape[1] - 1 + d]
    g0 = cols(rows(1) - rows(-1), -1) + 2 * cols(rows(1) - rows(-1), 0) + cols(rows(1) - rows(-1), 1)
    dc = cols(p, 1) - cols(p, -1)
    g1 = dc[:-2] + 2 * dc[1:-1] + dc[2:]
    return np.hypot(g0.astype(np.float32), g1.astype(np.float32))


def text_mask(frames, start, nframes=150, chunk=10, edge_percentile=90, max_std=1.5, dilate=4):
    """
    TEST INFRASTRUCTURE. The restatement of auto_slip.text_mask (auto_slip.py:81-94): the per-pixel
    population standard deviation of each chunk of frames (exact integer sums), its median over the
    chunks; the Sobel magnitude of frame start; strong (above the percentile) and steady (below
    max_std) pixels, dilated `dilate` times by the 3 x 3 cross, then every background region that
    does not touch the border (4-connected) filled.
    """
    f = np.asarray(frames)
    sd = chunk_std_median(f, start, nframes, chunk)
    edge = _sobel_magnitude(f[start].astype(np.float32))
    return mask_from_maps(edge, sd, edge_percentile, max_std, dilate)


def chunk_std_median(frames, start, nframes=150, chunk=10):
    """
    TEST INFRASTRUCTURE. The steadiness map of auto_slip.text_mask (auto_slip.py:87-90): per pixel,
    the population standard deviation of each chunk of `chunk` frames from `start` (exact integer
    sums, float32 result), then the median over the chunks (float32).
    """
    f = np.asarray(frames)
    stds = []
    for a in range(start, min(start + nframes, len(f)) - chunk + 1, chunk):
        x = f[a:a + chunk].astype(np.int64)
        s1, s2 = x.sum(0), (x * x).sum(0)
        var = (chunk * s2 - s1 * s1) / float(chunk * chunk)
        stds.append(np.sqrt(np.maximum(var, 0)).astype(np.float32))
    return np.median(np.stack(stds), axis=0)


def mask_from_maps(edge, sd, edge_percentile=90, max_std=1.5, dilate=4):
    """
    TEST INFRASTRUCTURE. The rest of auto_slip.text_mask (auto_slip.py:92-94) from the float32 edge
    magnitude and steadiness maps: pixels above numpy.percentile(edge, edge_percentile) and below
    max_std, dilated `dilate` times by the 3 x 3 cross (dilate < 1: until nothing changes, as
    scipy.ndimage.binary_dilation does), then every background region that does not touch the border
    (4-connected) filled.
    """
    from scipy import ndimage
    m = (edge > np.percentile(edge, edge_percentile)) & (sd < max_std)
    if dilate < 1:   # scipy repeats the dilation until nothing changes: the whole frame if any pixel is set
        m = np.ones_like(m) if m.any() else m
    for _ in range(dilate):
        g = m.copy()
        g[1:] |= m[:-1]
        g[:-1] |= m[1:]
        g[:, 1:] |= m[:, :-1]
        g[:, :-1] |= m[:, 1:]
        m = g
    labels, _ = ndimage.label(~m)   # 4-connected background regions
    border = np.unique(np.concatenate([labels[0], labels[-1], labels[:, 0], labels[:, -1]]))
    outside = np.isin(labels, border[border > 0])
    return ~outside


def ncc_peak(template, search):
    """
    TEST INFRASTRUCTURE. The restatement of stabilize.ncc_peak (python/slipcam/stabilize.py:22-44):
    the normalized correlation of the zero-mean template at every placement inside search (the
    products by FFT in float64, the box sums of the search exactly by cumulative sums; the variance
    floored at 1e-6), its largest value (the first if equal), a parabola per axis through it and its
    neighbours (no refinement at the edge or for a denominator below 1e-12), as (dy, dx) from the
    centre of the placements, and the value. A flat template gives (NaN, NaN, 0).
    """
    t = np.asarray(template, np.float64)
    s = np.asarray(search, np.float64)
    t0 = t - t.mean()
    tn = np.sqrt((t0 * t0).sum())
    if tn < 1e-6:
        return np.nan, np.nan, 0.0
    th, tw = t.shape
    H, W = s.shape
    num = np.fft.irfft2(np.fft.rfft2(s) * np.conj(np.fft.rfft2(t0, s=(H, W))), s=(H, W))[:H - th + 1, :W - tw + 1]

    def box(a):
        c = np.zeros((H + 1, W + 1))
        c[1:, 1:] = a.cumsum(0).cumsum(1)
        return c[th:, tw:] - c[:-th, tw:] - c[th:, :-tw] + c[:-th, :-tw]
    ssum, ssq = box(s), box(s * s)
    ncc = num / (np.sqrt(np.maximum(ssq - ssum * ssum / t.size, 1e-6)) * tn)
    i, j = np.unravel_index(int(np.argmax(ncc)), ncc.shape)

    def vertex(c, m, p):
        den = m - 2 * c + p
        return 0.0 if abs(den) < 1e-12 else 0.5 * (m - p) / den
    di = vertex(ncc[i, j], ncc[i - 1, j], ncc[i + 1, j]) if 0 < i < ncc.shape[0] - 1 else 0.0
    dj = vertex(ncc[i, j], ncc[i, j - 1], ncc[i, j + 1]) if 0 < j < ncc.shape[1] - 1 else 0.0
    return i + di - (ncc.shape[0] - 1) / 2, j + dj - (ncc.shape[1] - 1) / 2, ncc[i, j]


def fit_camera(dx, dy, x, y, iterations=3):
    """
    TEST INFRASTRUCTURE. The restatement of slip_series.fit_camera (python/slipcam/slip_series.py:
    49-72), similarity model: least squares of dx = p - a y + s x, dy = q + a x + s y over the points
    with both offsets finite, `iterations` times, each time dropping the points whose residual, in
    either component, is not below max(3 x 1.4826 x the median absolute deviation of the residuals
    in use, 0.3); NaN and 0 when fewer than 4 points are left at the start of a round. Returns the
    last fit and the number of points left after the last round.
    """
    dx, dy, x, y = (np.asarray(v, np.float64) for v in (dx, dy, x, y))
    use = np.isfinite(dx) & np.isfinite(dy)
    m = np.full(4, np.nan)
    for _ in range(iterations):
        if use.sum() < 4:
            return np.full(4, np.nan), 0
        k = np.flatnonzero(use)
        G = np.vstack([np.column_stack([np.ones(len(k)), np.zeros(len(k)), -y[k], x[k]]),
                       np.column_stack([np.zeros(len(k)), np.ones(len(k)), x[k], y[k]])])
        m = np.linalg.lstsq(G, np.concatenate([dx[k], dy[k]]), rcond=None)[0]
        rx = dx[k] - (m[0] - m[2] * y[k] + m[3] * x[k])
        ry = dy[k] - (m[1] + m[2] * x[k] + m[3] * y[k])
        r = np.concatenate([rx, ry])
        thr = max(3 * 1.4826 * np.median(np.abs(r - np.median(r))), 0.3)
        use[k] = (np.abs(rx) < thr) & (np.abs(ry) < thr)
    return m, int(use.sum())


def coarse_track(frames, ref, text, window=96, step=96, search=32, min_peak=0.5, start=0):
    """
    TEST INFRASTRUCTURE. The restatement of stabilize.coarse_track (python/slipcam/stabilize.py:
    54-96): the grid of window x window templates of the reference frame centred `search + half`
    pixels or more inside it, `step` apart, without those that touch the text mask or whose
    standard deviation is 2 or less; each frame, forward from ref then backward to start, searched
    +-search pixels around each template's position predicted by the previous frame's similarity
    transform (rounded half to even), the peaks of at least min_peak fitted by fit_camera. Returns
    (frames x 4 transforms, windows per fit, templates in use).
    """
    f = np.asarray(frames)
    n, h, w = f.shape
    half = window // 2
    ys = np.arange(search + half, h - search - half, step)
    xs = np.arange(search + half, w - search - half, step)
    cy, cx = (v.ravel() for v in np.meshgrid(ys, xs, indexing='ij'))
    refimg = f[ref].astype(np.float64)
    text = np.asarray(text, bool)
    sel = [not text[a - half:a + half, b - half:b + half].any() and refimg[a - half:a + half, b - half:b + half].std() > 2
           for a, b in zip(cy, cx)]
    sel = np.asarray(sel, bool)
    cy, cx = cy[sel], cx[sel]
    X, Y = cx - w / 2, cy - h / 2
    L = window + 2 * search
    params = np.full((n, 4), np.nan)
    used = np.zeros(n, int)
    params[ref], used[ref] = 0, len(cx)
    for frames_in_order in (range(ref + 1, n), range(ref - 1, start - 1, -1)):
        prev = np.zeros(4)
        for k in frames_in_order:
            img = f[k].astype(np.float64)
            px = X + prev[0] - prev[2] * Y + prev[3] * X + w / 2
            py = Y + prev[1] + prev[2] * X + prev[3] * Y + h / 2
            dx, dy = np.full(len(cx), np.nan), np.full(len(cx), np.nan)
            for t in range(len(cx)):
                top, left = int(np.rint(py[t])) - half - search, int(np.rint(px[t])) - half - search
                if top < 0 or left < 0 or top + L > h or left + L > w:
                    continue
                oy, ox, pk = ncc_peak(refimg[cy[t] - half:cy[t] + half, cx[t] - half:cx[t] + half],
                                      img[top:top + L, left:left + L])
                if pk >= min_peak:
                    dx[t] = (left + search + half + ox) - w / 2 - X[t]
                    dy[t] = (top + search + half + oy) - h / 2 - Y[t]
            fit, nfit = fit_camera(dx, dy, X, Y)
            if np.all(np.isfinite(fit)):
                params[k], used[k], prev = fit, nfit, fit
            else:
                params[k], used[k] = prev, 0
    return params, used, len(cx)


def _box_mean_1d(x, size, axis):
    """the box mean over `size` along `axis`, borders reflected (half-sample), float32 results from
    the window sums in float64 (exact for these values) divided by size"""
    x = np.moveaxis(np.asarray(x, np.float32), axis, -1).astype(np.float64)
    n = x.shape[-1]
    s1 = size // 2
    idx = np.arange(-s1, n + size - s1 - 1)
    idx = np.mod(idx, 2 * n)
    idx = np.where(idx < n, idx, 2 * n - 1 - idx)
    ext = x[..., idx]
    c = np.concatenate([np.zeros(x.shape[:-1] + (1,)), np.cumsum(ext, -1)], -1)
    out = ((c[..., size:size + n] - c[..., :n]) / size).astype(np.float32)
    return np.moveaxis(out, -1, axis)


def box_mean(x, size=31):
    """
    TEST INFRASTRUCTURE. The restatement of scipy.ndimage.uniform_filter(x, size) on a float32 image
    as stabilize.py:116-120 uses it: along axis 0, rounded to float32, then along axis 1.
    """
    return _box_mean_1d(_box_mean_1d(x, size, 0), size, 1)


def bilinear(img, cy, cx, cval):
    """map_coordinates(img, [cy, cx], order=1, mode='constant', cval): float64 weights, a coordinate
    outside [0, n - 1] (or NaN) taking cval, the result rounded to float32"""
    img = np.asarray(img, np.float32).astype(np.float64)
    h, w = img.shape
    cy, cx = np.asarray(cy, np.float64), np.asarray(cx, np.float64)
    inside = (cy >= 0) & (cy <= h - 1) & (cx >= 0) & (cx <= w - 1)
    y = np.where(inside, cy, 0.0)
    x = np.where(inside, cx, 0.0)
    y0, x0 = np.floor(y), np.floor(x)
    ty, tx = y - y0, x - x0
    y0, x0 = y0.astype(np.int64), x0.astype(np.int64)
    y1, x1 = np.minimum(y0 + 1, h - 1), np.minimum(x0 + 1, w - 1)
    v = (img[y0, x0] * (1 - ty) * (1 - tx) + img[y0, x1] * (1 - ty) * tx
         + img[y1, x0] * ty * (1 - tx) + img[y1, x1] * ty * tx)
    return np.where(inside, v, np.float64(np.float32(cval))).astype(np.float32)


def warp(frame, params, fill=None):
    """
    TEST INFRASTRUCTURE. The restatement of stabilize.warp (python/slipcam/stabilize.py:99-106): each
    pixel (x, y) of the reference takes the frame's value at the similarity transform of (x, y)
    about the image centre, bilinear, outside the frame the fill (default numpy's mean of the frame).
    """
    f = np.asarray(frame)
    h, w = f.shape
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    x, y = xx - w / 2, yy - h / 2
    p, q, a, s = np.asarray(params, np.float64)
    sx = x + p - a * y + s * x
    sy = y + q + a * x + s * y
    fill = f.mean() if fill is None else fill
    return bilinear(f.astype(np.float32), sy + h / 2, sx + w / 2, fill)


def stabilize(frames, params, text, size=31):
    """
    TEST INFRASTRUCTURE. The restatement of stabilize.stabilize (python/slipcam/stabilize.py:109-124):
    per frame, the text pixels replaced by the box mean of the pixels without text around them
    (divided by the box mean of the mask, floored at 1e-3; the mean of the frame's pixels without
    text where that mean is 1e-3 or less), warped onto the reference, clipped and cast to uint8;
    and the union of the warped text masks above 0.5.
    """
    f_all = np.asarray(frames)
    n, h, w = f_all.shape
    text = np.asarray(text, bool)
    keep = (~text).astype(np.float32)
    den = box_mean(keep, size)
    out = np.empty((n, h, w), np.uint8)
    union = np.zeros((h, w), bool)
    floor = np.float32(1e-3)
    for k in range(n):
        f = f_all[k].astype(np.float32)
        if text.any():
            local = box_mean(f * keep, size) / np.maximum(den, floor)
            f = np.where(text, np.where(den > floor, local, f[~text].mean()), f)
        out[k] = np.clip(warp(f, params[k]), 0, 255).astype(np.uint8)
        union |= warp(text.astype(np.float32), params[k], fill=0) > 0.5
    return out, union
