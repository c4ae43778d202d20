"""
The differentiable path (slipcam_b200.diff): float frames, a continuous shift per pair, the
hand-written adjoints of the surface and of the sub-pixel offsets.

CPU: the float64 torch restatement (diff_f64) against FP64 central finite differences (h = 1e-3)
and against the FP64 direct oracle. GPU: the CUDA forward against the float64 restatement and
against the uint8 correlation; the CUDA adjoints against the float64 autograd gradients (1e-4
relative); the refinement (1025 windows to 0.005 px) and the noise sensitivity against cov.
"""

import numpy as np
import pytest
import torch

import diff_f64 as ref
from oracle import oracle
from slipcam_b200 import framecor, synth

GRAD_TOL = 1e-4   # relative error of a gradient vector: |g - g_ref| / |g_ref|


def small_case(n=2, seed=0):
    """48 x 48 float frames, window 8, search 3 (L 14, M 7), a 2 x 2 grid, shifts in (-1, 1)."""
    rng = np.random.default_rng(seed)
    tex = synth.texture(64, 64, 1.5, rng)
    mover = synth.Mover(tex)
    frames = np.stack([mover.shifted(0.4 * k, -0.3 * k)[:48, :48] for k in range(n)]).astype(np.float32)
    ref_frame = mover.shifted(0.0, 0.0)[:48, :48].astype(np.float32)
    down, across = np.array([12, 26]), np.array([13, 25])
    shift = rng.uniform(-0.9, 0.9, (n, 2, 2, 2))
    shift[np.abs(shift - np.round(shift)) < 0.05] += 0.1   # away from the cubic's knots
    return dict(frames=frames, ref=ref_frame, down=down, across=across, W=8, R=3, shift=shift)


def f64_loss(c, frames, shift, G):
    r0, norms = ref.reference_windows(c['ref'], c['down'], c['across'], c['W'])
    rho = ref.surfaces(ref.chips(frames, shift, c['down'], c['across'], c['W'], c['R']), r0, norms, c['W'])
    return (rho * G).sum(), rho


# ---- CPU: the float64 restatement itself

def test_f64_gradient_matches_finite_differences():
    c = small_case()
    frames = torch.tensor(c['frames'], dtype=torch.float64, requires_grad=True)
    shift = torch.tensor(c['shift'], dtype=torch.float64, requires_grad=True)
    G = torch.as_tensor(np.random.default_rng(1).standard_normal((2, 2, 2, 7, 7)))
    loss, _ = f64_loss(c, frames, shift, G)
    gf, gs = torch.autograd.grad(loss, (frames, shift))
    h = 1e-3
    rng = np.random.default_rng(2)
    for _ in range(3):   # directional derivatives along random pixel directions
        d = torch.as_tensor(rng.standard_normal(frames.shape))
        with torch.no_grad():
            lp, _ = f64_loss(c, frames + h * d, shift, G)
            lm, _ = f64_loss(c, frames - h * d, shift, G)
        fd = (lp - lm) / (2 * h)
        an = (gf * d).sum()
        assert abs(fd - an) <= 1e-6 * abs(an) + 1e-9, (fd, an)
    for idx in [(0, 0, 0, 0), (0, 1, 1, 1), (1, 0, 1, 0), (1, 1, 0, 1)]:   # shift coordinates
        d = torch.zeros_like(shift)
        d[idx] = 1.0
        with torch.no_grad():
            lp, _ = f64_loss(c, frames, shift + h * d, G)
            lm, _ = f64_loss(c, frames, shift - h * d, G)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - gs[idx]) <= 1e-5 * abs(gs[idx]) + 1e-7, (idx, fd, gs[idx])


def test_f64_surface_matches_oracle_at_integer_shifts():
    """At shift 0 on uint8-valued frames the restatement is the reference's surface (FP64 oracle)."""
    c = small_case()
    frames = np.rint(c['frames']).astype(np.uint8)
    refu = np.rint(c['ref']).astype(np.uint8)
    o = oracle.correlate(48, 48, c['down'], c['across'], refu, frames, None, window=8, search=3, mode='f64',
                         surfaces=True)
    r0, norms = ref.reference_windows(refu.astype(np.float64), c['down'], c['across'], 8)
    rho = ref.surfaces(ref.chips(frames.astype(np.float64), torch.zeros((2, 2, 2, 2), dtype=torch.float64),
                                 c['down'], c['across'], 8, 3), r0, norms, 8)
    assert np.abs(rho.numpy() - o['surface']).max() < 1e-9


def test_f64_offsets_follow_the_reference_estimator():
    c = small_case()
    frames = np.rint(c['frames']).astype(np.uint8)
    refu = np.rint(c['ref']).astype(np.uint8)
    o = oracle.correlate(48, 48, c['down'], c['across'], refu, frames, None, window=8, search=3, mode='f64')
    r0, norms = ref.reference_windows(refu.astype(np.float64), c['down'], c['across'], 8)
    z = torch.zeros((2, 2, 2, 2), dtype=torch.float64)
    rho = ref.surfaces(ref.chips(frames.astype(np.float64), z, c['down'], c['across'], 8, 3), r0, norms, 8)
    off = ref.offsets(rho, z, 3).numpy()
    assert np.allclose(off, o['offsets64'], atol=1e-9, equal_nan=True)


# ---- GPU: the CUDA forward and adjoints

def cuda_case(c, device='cuda'):
    from slipcam_b200 import diff
    h, w = c['frames'].shape[1:]
    dc = diff.DiffCorrelator(h, w, c['down'], c['across'], window=c['W'], search=c['R'])
    dc.set_reference(torch.as_tensor(c['ref']))
    return dc


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.gpu
def test_cuda_surface_matches_f64():
    c = small_case()
    dc = cuda_case(c)
    fwd = dc.forward(torch.as_tensor(c['frames']), torch.as_tensor(c['shift'], dtype=torch.float32))
    _, rho = f64_loss(c, torch.tensor(c['frames'], dtype=torch.float64),
                      torch.tensor(c['shift'], dtype=torch.float32).double(), torch.zeros(1))
    assert np.abs(fwd['surface'].cpu().numpy() - rho.numpy()).max() < 2e-5


@pytest.mark.gpu
def test_cuda_surface_adjoint_matches_f64():
    c = small_case()
    dc = cuda_case(c)
    G = np.random.default_rng(3).standard_normal((2, 2, 2, 7, 7))
    frames = torch.tensor(c['frames'], device='cuda', requires_grad=True)
    shift = torch.tensor(c['shift'], dtype=torch.float32, device='cuda', requires_grad=True)
    loss = (dc.surface(frames, shift) * torch.as_tensor(G, dtype=torch.float32, device='cuda')).sum()
    gf, gs = torch.autograd.grad(loss, (frames, shift))
    frames64 = torch.tensor(c['frames'], dtype=torch.float64, requires_grad=True)
    shift64 = torch.tensor(c['shift'], dtype=torch.float32).double().requires_grad_(True)
    l64, _ = f64_loss(c, frames64, shift64, torch.as_tensor(G))
    rf, rs = torch.autograd.grad(l64, (frames64, shift64))
    assert rel(gf.cpu(), rf) < GRAD_TOL
    assert rel(gs.cpu(), rs) < GRAD_TOL


@pytest.mark.gpu
def test_cuda_offset_adjoint_matches_f64():
    c = small_case(seed=5)
    dc = cuda_case(c)
    frames = torch.tensor(c['frames'], device='cuda', requires_grad=True)
    shift = torch.tensor(c['shift'], dtype=torch.float32, device='cuda', requires_grad=True)
    off = dc.offsets(frames, shift)
    wts = torch.as_tensor(np.random.default_rng(4).standard_normal((2, 2, 2, 2)), dtype=torch.float32, device='cuda')
    ok = torch.isfinite(off)
    gf, gs = torch.autograd.grad((torch.where(ok, off, 0) * wts).sum(), (frames, shift))
    frames64 = torch.tensor(c['frames'], dtype=torch.float64, requires_grad=True)
    shift64 = torch.tensor(c['shift'], dtype=torch.float32).double().requires_grad_(True)
    r0, norms = ref.reference_windows(c['ref'], c['down'], c['across'], 8)
    rho = ref.surfaces(ref.chips(frames64, shift64, c['down'], c['across'], 8, 3), r0, norms, 8)
    off64 = ref.offsets(rho, shift64, 3)
    assert np.allclose(off.detach().cpu().numpy(), off64.detach().numpy(), atol=1e-4, equal_nan=True)
    ok64 = torch.isfinite(off64)
    rf, rs = torch.autograd.grad((torch.where(ok64, off64, 0) * wts.cpu().double()).sum(), (frames64, shift64))
    assert rel(gf.cpu(), rf) < GRAD_TOL
    assert rel(gs.cpu(), rs) < GRAD_TOL


@pytest.mark.gpu
def test_cuda_forward_matches_uint8_correlation():
    """At shift 0 on uint8-valued float frames the differentiable forward is the correlation."""
    frames, motion = synth.small(n=4)[:2]
    frames = np.asarray(frames)
    h, w = frames.shape[1:]
    down, across = framecor.window_grid(h, w, 32, 16, 16)
    cor = framecor.Correlator(h, w, down, across, window=32, search=16, backend='b200')
    cor.set_reference(frames[0])
    plain = cor.correlate(torch.as_tensor(frames).cuda(), surfaces=True)
    from slipcam_b200 import diff
    dc = diff.DiffCorrelator(h, w, down, across, window=32, search=16)
    dc.set_reference(torch.as_tensor(frames[0]).float())
    fwd = dc.forward(torch.as_tensor(frames).float())
    valid = (fwd['peak_at'] >= 0).cpu().numpy()
    assert valid.mean() > 0.8
    s1, s2 = plain['surface'].cpu().numpy()[valid], fwd['surface'].cpu().numpy()[valid]
    assert np.abs(s1 - s2).max() < 1e-5
    o1, o2 = plain['offsets'].cpu().numpy()[valid], fwd['offsets'].cpu().numpy()[valid]
    assert np.nanmax(np.abs(o1 - o2)) < 1e-3


@pytest.mark.gpu
def test_refinement_reaches_5_millipixels():
    """1025 windows (41 moved 256 x 256 float frames x 25 windows, shifts U[-3, 3]) refined to
    within 0.005 px of the true shift; the reference's own estimator is far coarser."""
    frames, shifts = synth.shifts_f32(n=42)
    down, across = framecor.window_grid(256, 256, 64, 8, 32)
    from slipcam_b200 import diff
    dc = diff.DiffCorrelator(256, 256, down, across, window=64, search=8)
    dc.set_reference(torch.as_tensor(frames[0]))
    r = dc.refine(torch.as_tensor(frames[1:]), iters=8)
    truth = shifts[1:, None, None, :]
    err = np.abs(r['offsets'].cpu().numpy() - truth).max(-1)
    err0 = np.abs(r['initial'].cpu().numpy() - truth).max(-1)
    assert err.size == 1025 and np.isfinite(err).all()
    assert err.max() <= 0.005, (err.max(), np.quantile(err, 0.99))
    assert np.median(err0) > 5 * np.median(err)


@pytest.mark.gpu
def test_noise_sensitivity_tracks_cov():
    """The offsets' covariance under pixel noise, J J^T sigma^2 from the adjoint: the variance the
    offsets show over noise draws, and correlated with the reported cov (a model from the peak's
    curvature and 1 - peak, which runs about ten times larger at 2 DN of noise)."""
    frames, shifts = synth.shifts_f32(n=9, noise=2.0, seed=7)
    down, across = framecor.window_grid(256, 256, 64, 8, 32)
    from slipcam_b200 import diff
    dc = diff.DiffCorrelator(256, 256, down, across, window=64, search=8)
    dc.set_reference(torch.as_tensor(frames[0]))
    sens = dc.sensitivity(torch.as_tensor(frames[1:])).cpu().numpy() * 2.0 ** 2
    cov = dc.forward(torch.as_tensor(frames[1:]))['cov'].cpu().numpy()
    ok = (sens[..., 0] > 0) & (cov[..., 0] < 99)
    assert ok.mean() > 0.9
    for c in range(2):
        ratio = sens[..., c][ok] / cov[..., c][ok]
        assert 0.01 < np.median(ratio) < 100, np.median(ratio)
        lr = np.corrcoef(np.log(sens[..., c][ok]), np.log(cov[..., c][ok]))[0, 1]
        assert lr > 0.3, lr
    # and it is the variance the offsets actually show over noise draws (Monte Carlo, 48 draws)
    rng = np.random.default_rng(11)
    draws = np.stack([dc.forward(torch.as_tensor(frames[1:] + rng.standard_normal(frames[1:].shape).astype(np.float32)
                                                 * 2.0))['offsets'].cpu().numpy() for _ in range(48)])
    var = draws.var(0)
    for c in range(2):
        assert 0.7 < np.median(sens[..., c][ok] / var[..., c][ok]) < 1.4
