"""
The differentiable correlation of float frames (b200 backend).

The normalized correlation surfaces and the sub-pixel offsets of framecor's Correlator, as torch
autograd functions of the frame pixels and of a continuous shift of every search window, with
hand-written CUDA adjoints (the math is stated in slipcam_b200/csrc/diff.h). Two uses are built on
them: a gradient-based continuous sub-pixel refinement of the offsets (``refine``) and the
pixel-noise sensitivity of the offsets (``sensitivity``), comparable with the reported ``cov``.

A pair's search window is sampled at its grid position + gross + shift with Keys' six-point cubic
convolution (fourth order, C1; the edge pixel repeats beyond the frame); at an integer shift that is the pixels
themselves, and the surface, peak, SNR and covariance are the reference's (cxx/cpu.cpp:115-160,
cxx/surface.h:30-146) on float pixels. A pair is invalid (NaN offsets, zero gradient) as in the
reference, with the floored position of its shifted window.

Everything runs on the GPU through the C ABI (include/slipcam_b200.h); there is no CPU path.
"""

import torch

from . import _lib, framecor


def _f32(x, device):
    return x.to(device=device, dtype=torch.float32).contiguous()


class DiffCorrelator:
    """Correlator(height, width, down, across, window=, search=, stat_size=) on float frames."""

    def __init__(self, height, width, down, across, *, window=64, search=48, stat_size=21, device=0):
        self.cor = framecor.Correlator(height, width, down, across, window=window, search=search,
                                       backend='b200', stat_size=stat_size, device=device)
        self.cor.set_form('fft32')   # the float frames' passes are the FP32 form's
        self.height, self.width = height, width
        self.ny, self.nx = self.cor.shape
        self.window, self.search = window, search
        self.L, self.M = window + 2 * search, 2 * search + 1
        self.device = torch.device('cuda', device)

    @property
    def shape(self):
        return self.ny, self.nx

    def _call(self, name, *args):
        _lib.raise_for(getattr(_lib.lib(), name)(self.cor._h, *args), self.cor._h)

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def set_reference(self, frame):
        """The reference frame (height x width), float32 (any real dtype is converted)."""
        f = _f32(torch.as_tensor(frame), self.device)
        if tuple(f.shape) != (self.height, self.width):
            raise ValueError('framecor: the reference frame must be height x width')
        self._call('b200_set_reference_f32_device', f.data_ptr(), self.width, self._stream())
        torch.cuda.current_stream(self.device).synchronize()

    def _inputs(self, frames, shift, gross):
        f = _f32(torch.as_tensor(frames), self.device)
        if f.dim() != 3 or tuple(f.shape[1:]) != (self.height, self.width):
            raise ValueError('framecor: the frames must be frames x height x width')
        n = f.shape[0]
        s = None
        if shift is not None:
            s = _f32(torch.as_tensor(shift), self.device)
            if tuple(s.shape) == (n, 2):
                s = s[:, None, None, :].expand(n, self.ny, self.nx, 2).contiguous()
            if tuple(s.shape) != (n, self.ny, self.nx, 2):
                raise ValueError('framecor: shift must be frames x 2 or frames x down x across x 2')
        g, mode = None, _lib.GROSS_NONE
        if gross is not None:
            g, mode = self.cor._gross(torch.as_tensor(gross), n, torch)
            g = g.to(self.device)
        return f, s, g, mode

    def _forward(self, f, s, g, mode):
        n, ny, nx, L, M = f.shape[0], self.ny, self.nx, self.L, self.M
        dev = self.device
        out = dict(chips=torch.empty((n, ny, nx, L, L), dtype=torch.float32, device=dev),
                   stats=torch.empty((n, ny, nx, M, M, 2), dtype=torch.float32, device=dev),
                   surface=torch.empty((n, ny, nx, M, M), dtype=torch.float32, device=dev),
                   peak_at=torch.empty((n, ny, nx), dtype=torch.int32, device=dev),
                   offsets=torch.empty((n, ny, nx, 2), dtype=torch.float32, device=dev),
                   peak=torch.empty((n, ny, nx), dtype=torch.float32, device=dev),
                   snr=torch.empty((n, ny, nx), dtype=torch.float32, device=dev),
                   cov=torch.empty((n, ny, nx, 3), dtype=torch.float32, device=dev))
        if n:
            self._call('b200_diff_forward', f.data_ptr(), n, self.width, None if g is None else g.data_ptr(), mode,
                       None if s is None else s.data_ptr(), out['chips'].data_ptr(), out['stats'].data_ptr(),
                       out['surface'].data_ptr(), out['peak_at'].data_ptr(), out['offsets'].data_ptr(),
                       out['peak'].data_ptr(), out['snr'].data_ptr(), out['cov'].data_ptr(), self._stream())
        if s is not None:
            out['offsets'] = out['offsets'] + s
        return out

    def _backward(self, f, s, g, mode, fwd, g_surface, frames_grad=True, shift_grad=True):
        n = f.shape[0]
        g_chips = torch.empty_like(fwd['chips'])
        g_frames = torch.zeros_like(f) if frames_grad else None
        g_shift = torch.empty((n, self.ny, self.nx, 2), dtype=torch.float32, device=self.device) if shift_grad else None
        if n:
            self._call('b200_diff_backward', f.data_ptr(), n, self.width, None if g is None else g.data_ptr(), mode,
                       None if s is None else s.data_ptr(), fwd['chips'].data_ptr(), fwd['stats'].data_ptr(),
                       fwd['surface'].data_ptr(), g_surface.contiguous().data_ptr(), g_chips.data_ptr(),
                       None if g_frames is None else g_frames.data_ptr(),
                       None if g_shift is None else g_shift.data_ptr(), self._stream())
        return g_chips, g_frames, g_shift

    def _offset_cotangent(self, fwd, g_offsets):
        n = fwd['surface'].shape[0]
        g_surface = torch.empty_like(fwd['surface'])
        if n:
            self._call('b200_offset_adjoint', n, fwd['surface'].data_ptr(), fwd['peak_at'].data_ptr(),
                       _f32(g_offsets, self.device).data_ptr(), g_surface.data_ptr(), self._stream())
        return g_surface

    def forward(self, frames, shift=None, gross=None):
        """Everything of the forward pass, without autograd: surface (n, ny, nx, M, M), offsets
        (the shift included), peak, snr, cov, peak_at (u M + v, -1 if invalid), chips, stats."""
        with torch.no_grad():
            return self._forward(*self._inputs(frames, shift, gross))

    def surface(self, frames, shift=None, gross=None):
        """The normalized surfaces (n, ny, nx, M, M), differentiable in frames and shift."""
        return _Surface.apply(frames, shift, self, gross)

    def offsets(self, frames, shift=None, gross=None):
        """The sub-pixel offsets (n, ny, nx, 2), shift included, differentiable in frames and shift."""
        return _Offsets.apply(frames, shift, self, gross)

    def refine(self, frames, gross=None, iters=6):
        """
        Continuous sub-pixel refinement of every pair's displacement d (down, across, relative to
        its gross position): the maximum of the normalized correlation as a continuous function
        of d, by Newton steps. At each step the search window is sampled at the fraction
        t = d - floor(d) (so it stays where the reference puts it) and the correlation is read at
        the integer point floor(d) + R of that surface: its gradient in t comes from the adjoint,
        its Hessian from the 3 x 3 quadratic fit around that point (cxx/surface.h:79-96). Starts
        at the reference's sub-pixel estimate.

        Returns a dict: offsets (n, ny, nx, 2) = gross + d, the initial (reference) offsets, and
        the last gradient norm per pair. Pairs without a valid interior peak keep the initial
        offsets.
        """
        f, _, g, mode = self._inputs(frames, None, gross)
        n, ny, nx, M, R = f.shape[0], self.ny, self.nx, self.M, self.search
        dev = self.device
        with torch.no_grad():
            fwd = self._forward(f, None, g, mode)
            gyx = torch.zeros((n, ny, nx, 2), dtype=torch.float32, device=dev)
            if g is not None:
                gyx = g.float() if g.dim() == 4 else g.float()[:, None, None, :].expand(n, ny, nx, 2)
            valid = (fwd['peak_at'] >= 0) & torch.isfinite(fwd['offsets']).all(-1)
            d = torch.where(valid[..., None], fwd['offsets'] - gyx, torch.zeros_like(gyx)).double()
            live = valid.clone()
            grad_norm = torch.zeros((n, ny, nx), dtype=torch.float32, device=dev)
            steps = torch.arange(-1, 2, device=dev)
            for _ in range(iters):
                fl = torch.floor(d)
                t = (d - fl).float().contiguous()
                uv = (fl + R).long()
                u1, v1 = uv[..., 0], uv[..., 1]
                live = live & (u1 >= 1) & (u1 <= M - 2) & (v1 >= 1) & (v1 <= M - 2)
                u1, v1 = u1.clamp(1, M - 2), v1.clamp(1, M - 2)
                onehot = torch.zeros((n, ny, nx, M * M), dtype=torch.float32, device=dev)
                onehot.scatter_(-1, (u1 * M + v1)[..., None], 1.0)
                onehot = onehot.view(n, ny, nx, M, M) * live[..., None, None]
                fw = self._forward(f, t, g, mode)
                _, _, gt = self._backward(f, t, g, mode, fw, onehot, frames_grad=False, shift_grad=True)
                s = fw['surface'].double()
                rows = torch.gather(s, 3, (u1[..., None] + steps)[..., :, None].expand(n, ny, nx, 3, M))
                p = torch.gather(rows, 4, (v1[..., None] + steps)[..., None, :].expand(n, ny, nx, 3, 3))
                c3 = (p[..., 0, :].sum(-1) + p[..., 2, :].sum(-1) - 2 * p[..., 1, :].sum(-1)) / 6
                c5 = (p[..., :, 0].sum(-1) + p[..., :, 2].sum(-1) - 2 * p[..., :, 1].sum(-1)) / 6
                c4 = (p[..., 2, 2] - p[..., 2, 0] - p[..., 0, 2] + p[..., 0, 0]) / 4
                hyy, hxy, hxx = 2 * c3, c4, 2 * c5
                det = hyy * hxx - hxy * hxy
                gd = gt.double()
                ok = live & (det > 0) & (hyy < 0) & torch.isfinite(gd).all(-1)
                sdet = torch.where(ok, det, torch.ones_like(det))
                dy = -(hxx * gd[..., 0] - hxy * gd[..., 1]) / sdet
                dx = -(-hxy * gd[..., 0] + hyy * gd[..., 1]) / sdet
                step = torch.stack([dy, dx], -1).clamp(-0.5, 0.5)
                d = torch.where(ok[..., None], d + step, d)
                grad_norm = torch.where(live, gt.norm(dim=-1), grad_norm)
            offsets = torch.where(live[..., None], gyx + d.float(), fwd['offsets'])
        return dict(offsets=offsets, initial=fwd['offsets'], grad_norm=grad_norm)

    def sensitivity(self, frames, gross=None):
        """
        The covariance of the offsets under independent unit-variance noise on the frame pixels,
        J J^T from the adjoint (J = d offsets / d pixels), per pair: (n, ny, nx, 3) as cov (down,
        across, cross); multiply by the noise variance. Zero for invalid and edge peaks.
        """
        f, _, g, mode = self._inputs(frames, None, gross)
        with torch.no_grad():
            fwd = self._forward(f, None, g, mode)
            jac = []
            for c in range(2):
                go = torch.zeros_like(fwd['offsets'])
                go[..., c] = 1.0
                gs = self._offset_cotangent(fwd, go)
                gc, _, _ = self._backward(f, None, g, mode, fwd, gs, frames_grad=False, shift_grad=False)
                jac.append(gc.double().flatten(-2))
            j0, j1 = jac
            return torch.stack([(j0 * j0).sum(-1), (j1 * j1).sum(-1), (j0 * j1).sum(-1)], -1).float()


class _Surface(torch.autograd.Function):
    @staticmethod
    def forward(ctx, frames, shift, dc, gross):
        f, s, g, mode = dc._inputs(frames, shift, gross)
        fwd = dc._forward(f, s, g, mode)
        ctx.dc, ctx.g, ctx.mode = dc, g, mode
        ctx.fwd = {k: fwd[k] for k in ('chips', 'stats', 'surface')}
        _remember(ctx, frames, shift)
        ctx.save_for_backward(f, s)
        return fwd['surface']

    @staticmethod
    def backward(ctx, g_surface):
        f, s = ctx.saved_tensors
        need_f, need_s = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        _, gf, gs = ctx.dc._backward(f, s, ctx.g, ctx.mode, ctx.fwd, g_surface, need_f, need_s)
        return _shaped(ctx, gf, gs)


class _Offsets(torch.autograd.Function):
    @staticmethod
    def forward(ctx, frames, shift, dc, gross):
        f, s, g, mode = dc._inputs(frames, shift, gross)
        fwd = dc._forward(f, s, g, mode)
        ctx.dc, ctx.g, ctx.mode = dc, g, mode
        ctx.fwd = {k: fwd[k] for k in ('chips', 'stats', 'surface', 'peak_at')}
        _remember(ctx, frames, shift)
        ctx.save_for_backward(f, s)
        return fwd['offsets']

    @staticmethod
    def backward(ctx, g_offsets):
        f, s = ctx.saved_tensors
        need_f, need_s = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        g_offsets = torch.nan_to_num(g_offsets.float())
        g_surface = ctx.dc._offset_cotangent(ctx.fwd, g_offsets)
        _, gf, gs = ctx.dc._backward(f, s, ctx.g, ctx.mode, ctx.fwd, g_surface, need_f, need_s)
        if need_s:   # offsets = (the sub-pixel estimate of the shifted window) + shift
            gs = gs + g_offsets * (ctx.fwd['peak_at'] >= 0)[..., None]
        return _shaped(ctx, gf, gs)


def _remember(ctx, frames, shift):
    ctx.frames_like = (torch.as_tensor(frames).dtype, torch.as_tensor(frames).device)
    ctx.shift_like = None if shift is None else (tuple(torch.as_tensor(shift).shape), torch.as_tensor(shift).dtype,
                                                 torch.as_tensor(shift).device)


def _shaped(ctx, gf, gs):
    """The cotangents in the caller's dtypes, devices and shapes (a per-frame shift sums its pairs)."""
    if gf is not None:
        gf = gf.to(dtype=ctx.frames_like[0], device=ctx.frames_like[1])
    if gs is not None and ctx.shift_like is not None:
        shape, dtype, device = ctx.shift_like
        if len(shape) == 2:
            gs = gs.sum((1, 2))
        gs = gs.to(dtype=dtype, device=device)
    return gf, gs, None, None
