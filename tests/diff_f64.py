"""
A float64 torch restatement of the differentiable correlation (slipcam_b200/csrc/diff.h), for the
tests: its autograd gradients are the reference the CUDA adjoints are checked against, and it is
itself checked against FP64 finite differences and the FP64 direct oracle. Test infrastructure
only (plain torch ops, CPU or GPU).

Per pair: chip = Keys six-point cubic sample of the frame at (down + gy - R + ty, across + gx - R + tx),
the edge pixel repeated beyond the frame;
c = the W x W reference window r0 (zero mean, double) correlated over the chip (M x M); rho = c /
(norm sqrt(S2 - S1^2 / n)) with the chip's box sums S1, S2; the offsets from the reference's 3 x 3
fit (cxx/surface.h:71-146), else a parabola per axis, plus gross + peak - R + t.
"""

import torch
import torch.nn.functional as F


def interp_weights(t):
    """Keys' six-point cubic convolution weights of the taps at -2 .. 3 for fractions t in [0, 1)."""
    def k1(x): return (4 / 3 * x - 7 / 3) * x * x + 1
    def k2(x): return ((-7 / 12 * x + 3) * x - 59 / 12) * x + 2.5
    def k3(x): return ((1 / 12 * x - 2 / 3) * x + 1.75) * x - 1.5
    return torch.stack([k3(t + 2), k2(t + 1), k1(t), k1(1 - t), k2(2 - t), k3(3 - t)], -1)


def reference_windows(ref, down, across, W):
    """r0 (nwin, W, W) float64 zero-mean windows of the reference frame and their norms."""
    ref = torch.as_tensor(ref, dtype=torch.float64)
    wins = torch.stack([ref[y:y + W, x:x + W] for y in down for x in across])
    r0 = wins - wins.mean((1, 2), keepdim=True)
    return r0, r0.square().sum((1, 2)).sqrt()


def chips(frames, shift, down, across, W, R, gross=None):
    """(n, ny, nx, L, L) float64 chips; shift (n, ny, nx, 2) float64 (may require grad)."""
    frames = torch.as_tensor(frames, dtype=torch.float64)
    n = frames.shape[0]
    ny, nx, L = len(down), len(across), W + 2 * R
    out = []
    for f in range(n):
        for yy in range(ny):
            for xx in range(nx):
                gy = gx = 0
                if gross is not None:
                    g = gross[f] if gross.ndim == 2 else gross[f, yy, xx]
                    gy, gx = int(g[0]), int(g[1])
                t = shift[f, yy, xx]
                fy, fx = torch.floor(t[0].detach()), torch.floor(t[1].detach())
                y0 = int(down[yy]) + gy - R + int(fy)
                x0 = int(across[xx]) + gx - R + int(fx)
                wy, wx = interp_weights(t[0] - fy), interp_weights(t[1] - fx)
                h, w = frames.shape[1:]
                cols = (torch.arange(L + 5) + x0 - 2).clamp(0, w - 1)   # the edge pixel repeats
                c = 0
                for d in range(6):
                    rows = frames[f][(torch.arange(L) + y0 - 2 + d).clamp(0, h - 1)][:, cols]
                    c = c + wy[d] * sum(wx[e] * rows[:, e:e + L] for e in range(6))
                out.append(c)
    return torch.stack(out).view(n, ny, nx, L, L)


def surfaces(ch, r0, norms, W):
    """rho (n, ny, nx, M, M) from chips (n, ny, nx, L, L) and the reference windows."""
    n, ny, nx, L, _ = ch.shape
    x = ch.reshape(n, ny * nx, L, L)
    c = torch.stack([F.conv2d(x[:, k:k + 1], r0[k][None, None]) for k in range(ny * nx)], 1)[:, :, 0]
    ones = torch.ones((1, 1, W, W), dtype=torch.float64, device=ch.device)
    s1 = F.conv2d(x.reshape(-1, 1, L, L), ones).view(c.shape)
    s2 = F.conv2d(x.reshape(-1, 1, L, L).square(), ones).view(c.shape)
    var_n = s2 - s1 * s1 / (W * W)
    safe = torch.where(var_n > 0, var_n, torch.ones_like(var_n))
    rho = torch.where(var_n > 0, c / (norms[None, :, None, None] * safe.sqrt()), torch.zeros_like(c))
    M = rho.shape[-1]
    return rho.view(n, ny, nx, M, M)


def subpixel(s, u, v):
    """(du, dv) of the reference's sub-pixel estimator at the peak (u, v) of one M x M surface s
    (float64 tensor; the branch is chosen on the values, the formula differentiates)."""
    M = s.shape[-1]
    zero = s.new_zeros(())
    if not (0 < u < M - 1 and 0 < v < M - 1):
        return zero, zero
    f = s[u - 1:u + 2, v - 1:v + 2]
    c1 = (f[2].sum() - f[0].sum()) / 6
    c2 = (f[:, 2].sum() - f[:, 0].sum()) / 6
    c3 = (f[0].sum() + f[2].sum() - 2 * f[1].sum()) / 6
    c5 = (f[:, 0].sum() + f[:, 2].sum() - 2 * f[:, 1].sum()) / 6
    c4 = (f[2, 2] - f[2, 0] - f[0, 2] + f[0, 0]) / 4
    det = 4 * c3 * c5 - c4 * c4
    if c3.item() < 0 and det.item() > 0:
        du = (c4 * c2 - 2 * c5 * c1) / det
        dv = (c4 * c1 - 2 * c3 * c2) / det
        if abs(du.item()) <= 1 and abs(dv.item()) <= 1:
            return du, dv

    def parabola(m, c, p):
        den = m - 2 * c + p
        return 0.5 * (m - p) / den if den.item() < 0 else zero

    return parabola(f[0, 1], f[1, 1], f[2, 1]), parabola(f[1, 0], f[1, 1], f[1, 2])


def offsets(rho, shift, R, gross=None):
    """(n, ny, nx, 2) offsets from the surfaces: gross + peak - R + sub-pixel + shift (NaN where
    the surface has no positive value)."""
    n, ny, nx, M, _ = rho.shape
    out = []
    for f in range(n):
        for yy in range(ny):
            for xx in range(nx):
                s = rho[f, yy, xx]
                at = int(torch.argmax(s.detach()).item())
                if not s.detach().flatten()[at] > 0:
                    out.append(torch.full((2,), float('nan'), dtype=torch.float64, device=rho.device))
                    continue
                u, v = divmod(at, M)
                du, dv = subpixel(s, u, v)
                gy = gx = 0
                if gross is not None:
                    g = gross[f] if gross.ndim == 2 else gross[f, yy, xx]
                    gy, gx = int(g[0]), int(g[1])
                out.append(torch.stack([gy + u - R + du + shift[f, yy, xx, 0], gx + v - R + dv + shift[f, yy, xx, 1]]))
    return torch.stack(out).view(n, ny, nx, 2)
