"""
Seeded synthetic video for the correlate workloads (the real slipcam videos are not distributed).

Every workload uses the same texture: N(0, 1) noise smoothed by a periodic Gaussian of sigma px,
rescaled to mean 128 and standard deviation 40, clipped to 0-255. A frame is that texture moved
by a sub-pixel Fourier shift (periodic), with an extra shift on the far side of a fault line,
plus Gaussian noise, rounded and clipped to uint8. The motion (down, across) is the motion of
the frame's content, i.e. what framecor reports as the offset.

Workloads (sizes as named):
  small      16 x 360 x 640, sigma 1.5, frame k moved by (0.3k, 0.2k) plus 0.5k across beyond the
             diagonal through the centre, noise 2 DN; window 32, search 16, skip 16; frame 0 is
             the reference
  hd         300 x 720 x 1280, sigma 2, camera random walk of 0.5 px steps, fault step ramping
             0 -> 40 px across over frames 100-130 along a line at 30 degrees, noise 2 DN;
             window 64, search 48, skip 16; per-frame gross = round(camera motion)
  mixed      64 x 720 x 1280 with 10 % flat (100 DN), 5 % saturated (255) and a box of 8-px
             stripes; grids 32/16, 64/48, 128/64 (skip 16); per-window gross U[-20, 20]
  stream     1000 x 1080 x 1920, sigma 2, noise 3 DN, a 5 Hz 4 px shake plus a random walk, a
             60 px fault step over 30 frames; window 64, search 64, skip 8
  camera     a camera moving over a textured scene (default 24 x 240 x 320; 720 x 1280 for the
             stabilize workload): frame k shows the scene through the similarity transform
             params[k] = (p, q, a, s) about the image centre (the content at x of the reference
             frame appears at x + p - a y + s x, y + q + a x + s y), a random walk from the
             reference frame, bicubic resampling, burned-in text boxes fixed in the frame, optional
             blank frames; for stabilize.coarse_track
  shifts_f32 float32 frames (default 41 x 256 x 256), sigma 2, frame k moved as a whole by a
             continuous shift U[-3, 3] px per axis (frame 0 unmoved: the reference), optional
             Gaussian noise, not rounded; window 64, search 8, skip 32 (the differentiable path)
"""

import math

import numpy as np


def _freqs(h, w):
    return np.fft.fftfreq(h)[:, None], np.fft.fftfreq(w)[None, :]


def texture(h, w, sigma, rng):
    """The smoothed, rescaled and clipped texture, float64 (h, w)."""
    ky, kx = _freqs(h, w)
    spec = np.fft.fft2(rng.standard_normal((h, w)))
    spec *= np.exp(-2.0 * math.pi ** 2 * sigma ** 2 * (ky ** 2 + kx ** 2))
    t = np.fft.ifft2(spec).real
    t = (t - t.mean()) / t.std() * 40.0 + 128.0
    return np.clip(t, 0.0, 255.0)


class Mover:
    """Sub-pixel Fourier shifts of one texture; numpy, or torch on a device when given."""

    def __init__(self, tex, device=None):
        self.h, self.w = tex.shape
        self.device = device
        if device is None:
            self.spec = np.fft.fft2(tex)
            ky, kx = _freqs(self.h, self.w)
            self.ky, self.kx = ky[:, 0], kx[0, :]
        else:
            import torch
            self.torch = torch
            t = torch.as_tensor(tex, dtype=torch.float64, device=device)
            self.spec = torch.fft.fft2(t)
            self.ky = torch.fft.fftfreq(self.h, dtype=torch.float64, device=device)
            self.kx = torch.fft.fftfreq(self.w, dtype=torch.float64, device=device)

    def shifted(self, dy, dx):
        """The texture with its content moved by (dy, dx) px (down, across)."""
        if self.device is None:
            ramp = np.exp(-2j * math.pi * self.ky * dy)[:, None] * np.exp(-2j * math.pi * self.kx * dx)[None, :]
            return np.fft.ifft2(self.spec * ramp).real
        torch = self.torch
        ry = torch.exp(-2j * math.pi * self.ky * dy)
        rx = torch.exp(-2j * math.pi * self.kx * dx)
        return torch.fft.ifft2(self.spec * (ry[:, None] * rx[None, :])).real


def _to_u8(img, noise, rng, device=None):
    if device is None:
        return np.clip(np.rint(img + rng.standard_normal(img.shape) * noise), 0, 255).astype(np.uint8)
    torch = __import__('torch')
    gen_noise = torch.as_tensor(rng.standard_normal(tuple(img.shape)).astype(np.float32), device=device)
    return torch.clamp(torch.round(img + gen_noise.double() * noise), 0, 255).to(torch.uint8)


def _side(h, w, angle_deg):
    """The far side of a line through the centre at angle_deg from the across axis."""
    y, x = np.mgrid[0:h, 0:w]
    a = math.radians(angle_deg)
    return (-(x - w / 2.0) * math.sin(a) + (y - h / 2.0) * math.cos(a)) > 0


def video(h, w, n, motion, step, *, sigma=2.0, noise=2.0, angle=None, seed=0, device=None):
    """n frames: frame k has content moved by motion[k] (down, across) plus step[k] across on
    the far side of the fault line (angle in degrees; the diagonal through the centre if None).
    Returns uint8 (n, h, w), numpy or a torch tensor on device."""
    rng = np.random.default_rng(seed)
    tex = texture(h, w, sigma, rng)
    mover = Mover(tex, device)
    if angle is None:
        angle = math.degrees(math.atan2(h, w))
    side = _side(h, w, angle)
    if device is not None:
        import torch
        side = torch.as_tensor(side, device=device)
        out = torch.empty((n, h, w), dtype=torch.uint8, device=device)
    else:
        out = np.empty((n, h, w), np.uint8)
    for k in range(n):
        dy, dx = float(motion[k][0]), float(motion[k][1])
        near = mover.shifted(dy, dx)
        if step[k] != 0:
            far = mover.shifted(dy, dx + float(step[k]))
            img = far * side + near * ~side if device is None else torch.where(side, far, near)
        else:
            img = near
        out[k] = _to_u8(img, noise, rng, device)
    return out


def small(n=16, h=360, w=640, seed=0, device=None):
    """The small workload: frames, motion (n, 2), step (n,)."""
    k = np.arange(n)
    motion = np.stack([0.3 * k, 0.2 * k], 1)
    step = 0.5 * k
    frames = video(h, w, n, motion, step, sigma=1.5, noise=2.0, seed=seed, device=device)
    return frames, motion, step


def hd(n=300, h=720, w=1280, seed=1, device=None, count=None):
    """The 720p workload: frames, camera motion (n, 2), fault step (n,), gross (n, 2) int32.
    count: render only the first count frames (the motion of all n is the same either way)."""
    rng = np.random.default_rng(seed + 1000)
    theta = rng.uniform(0, 2 * math.pi, n)
    steps = 0.5 * np.stack([np.sin(theta), np.cos(theta)], 1)
    steps[0] = 0
    motion = np.cumsum(steps, 0)
    k = np.arange(n)
    step = 40.0 * np.clip((k - 100) / 30.0, 0.0, 1.0)
    m = n if count is None else min(count, n)
    frames = video(h, w, m, motion, step, sigma=2.0, noise=2.0, angle=30.0, seed=seed, device=device)
    gross = np.rint(motion).astype(np.int32)
    return frames, motion, step, gross


def stream(n=1000, h=1080, w=1920, seed=2, device=None, count=None):
    """The 1080p streaming workload: frames, motion, step, gross (n, 2) int32. count: render only the
    first count frames (the motion of all n is the same either way)."""
    rng = np.random.default_rng(seed + 1000)
    t = np.arange(n) / 30.0
    walk = np.cumsum(rng.normal(0, 0.3, (n, 2)), 0)
    shake = 4.0 * np.stack([np.sin(2 * math.pi * 5 * t), np.cos(2 * math.pi * 5 * t + 0.7)], 1)
    motion = walk + shake
    k = np.arange(n)
    step = 60.0 * np.clip((k - n // 2) / 30.0, 0.0, 1.0)
    m = n if count is None else min(count, n)
    frames = video(h, w, m, motion, step, sigma=2.0, noise=3.0, angle=30.0, seed=seed, device=device)
    return frames, motion, step, np.rint(motion).astype(np.int32)


def mixed(n=64, h=720, w=1280, seed=3):
    """The uneven-work workload (numpy): frames with flat, saturated and striped regions."""
    rng = np.random.default_rng(seed + 1000)
    motion = np.cumsum(rng.normal(0, 0.3, (n, 2)), 0)
    frames = video(h, w, n, motion, np.zeros(n), sigma=2.0, noise=2.0, seed=seed)
    flat = (slice(0, int(0.10 * h)), slice(0, w))             # 10 % of the area
    sat = (slice(h - int(0.05 * h), h), slice(0, w))          # 5 %
    frames[:, flat[0], flat[1]] = 100
    frames[:, sat[0], sat[1]] = 255
    y0, x0 = h // 3, w // 3
    stripes = (128 + 60 * np.sin(2 * math.pi * np.arange(256) / 8.0)).astype(np.uint8)
    frames[:, y0:y0 + 160, x0:x0 + 256] = stripes[None, None, :]
    return frames, motion


def shifts_f32(n=41, h=256, w=256, seed=4, noise=0.0, max_shift=3.0):
    """Float frames moved by continuous shifts: frames (n, h, w) float32, shifts (n, 2) float64
    (down, across; shifts[0] = 0). Noise (DN, Gaussian) is added to every frame but the first."""
    rng = np.random.default_rng(seed + 1000)
    mover = Mover(texture(h, w, 2.0, rng))
    shifts = rng.uniform(-max_shift, max_shift, (n, 2))
    shifts[0] = 0.0
    frames = np.empty((n, h, w), np.float32)
    for k in range(n):
        img = mover.shifted(*shifts[k])
        if k and noise:
            img = img + rng.standard_normal(img.shape) * noise
        frames[k] = img
    return frames, shifts


def camera(n=24, h=240, w=320, *, ref=0, seed=6, sigma=2.0, noise=1.0, walk=(2.0, 2.0, 0.003, 0.003),
           text=((40, 8, 200, 24),), flat=None, blank=(), device=None):
    """A camera moving over a textured scene. Returns frames (n, h, w) uint8 (a CUDA tensor when
    device is given), params (n, 4) float64 (params[ref] = 0, a random walk of steps N(0, walk)
    away from it both ways) and the text mask (h, w) bool. text: boxes (x0, y0, x1, y1) drawn in
    every frame at the same place (a bright outline around dark strokes); flat: a box (x0, y0, x1,
    y1) of the scene made uniform (100 DN); blank: frames replaced by a uniform 128 DN."""
    rng = np.random.default_rng(seed)
    pad = 64 + int(4 * max(walk[0], walk[1]) * math.sqrt(n))
    tex = texture(h + 2 * pad, w + 2 * pad, sigma, rng)
    if flat is not None:
        x0, y0, x1, y1 = flat
        tex[y0 + pad:y1 + pad, x0 + pad:x1 + pad] = 100.0
    steps = rng.normal(0.0, 1.0, (n, 4)) * np.asarray(walk, np.float64)
    params = np.zeros((n, 4))
    for k in range(ref + 1, n):
        params[k] = params[k - 1] + steps[k]
    for k in range(ref - 1, -1, -1):
        params[k] = params[k + 1] + steps[k]
    mask = np.zeros((h, w), bool)
    for x0, y0, x1, y1 in text:
        mask[y0:y1, x0:x1] = True
    if device is None:
        from scipy import ndimage
        coef = ndimage.spline_filter(tex, order=3)
        yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
        yy -= h / 2
        xx -= w / 2
    else:
        import torch
        t = torch.as_tensor(tex, dtype=torch.float32, device=device)[None, None]
        yy, xx = torch.meshgrid(torch.arange(h, device=device, dtype=torch.float64) - h / 2,
                                torch.arange(w, device=device, dtype=torch.float64) - w / 2, indexing='ij')
    frames = np.empty((n, h, w), np.uint8)
    for k in range(n):
        p, q, a, s = params[k]
        # the scene point seen at frame pixel z: the inverse of z = (1 + s, -a; a, 1 + s) x + (p, q)
        det = (1 + s) ** 2 + a ** 2
        zx, zy = xx - p, yy - q
        sx = ((1 + s) * zx + a * zy) / det + w / 2 + pad
        sy = (-a * zx + (1 + s) * zy) / det + h / 2 + pad
        if device is None:
            img = ndimage.map_coordinates(coef, [sy, sx], order=3, mode='nearest', prefilter=False)
        else:
            import torch
            g = torch.stack([sx / (w + 2 * pad - 1) * 2 - 1, sy / (h + 2 * pad - 1) * 2 - 1], -1)
            img = torch.nn.functional.grid_sample(t, g[None].float(), mode='bicubic', padding_mode='border',
                                                  align_corners=True)[0, 0].double().cpu().numpy()
        if noise:
            img = img + rng.standard_normal((h, w)) * noise
        for x0, y0, x1, y1 in text:
            img[y0:y1, x0:x1] = 30.0
            img[y0:y0 + 2, x0:x1] = img[y1 - 2:y1, x0:x1] = 240.0
            img[y0:y1, x0:x0 + 2] = img[y0:y1, x1 - 2:x1] = 240.0
            img[y0 + 4:y1 - 4:4, x0 + 4:x1 - 4] = 220.0
        if k in blank:
            img = np.full((h, w), 128.0)
        frames[k] = np.clip(np.rint(img), 0, 255).astype(np.uint8)
    if device is not None:
        import torch
        return torch.as_tensor(frames).to(device), params, mask
    return frames, params, mask
