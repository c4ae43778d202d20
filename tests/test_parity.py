"""
Parity of the b200 backend (through its C ABI) with the reference and the oracle, on the GPU:

* the reference's own CPU backend (tests/golden fixtures): the same invalid windows, offsets
  within 1e-3 px except documented near-ties, peak within 1e-4, SNR within 1e-2 relative (the
  reference test's CPU/CUDA agreement bounds, cxx tests/test_framecor.py:92-94);
* the FP64 oracle: offsets within 0.01 px, SNR within 1e-3 relative, integer peaks identical except
  near-ties (the two best shifts within 1e-5 of each other on the FP64 surface);
* the summed-area tables: bit-exact against the oracle's int64 tables (the 32-bit sum table modulo
  2^32);
* the normalized surfaces against the oracle's float restatement, 2e-5 absolute;
* per-frame gross == the same gross per window, bit for bit; device tensors == host arrays.
"""

import numpy as np
import pytest

import cases
from oracle import oracle
from slipcam_b200 import framecor, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')

SUPPORTED = list(cases.NAMES)   # 'big' (window 128 + search 64, L = 256) runs the staged big transform
NEAR_TIE = 1e-5
TC_NEAR_TIE = 2e-3   # a near-tie for the FP16 tensor-core form: within a few times its surface error (3e-4)


def golden(name):
    return dict(np.load(f'{cases.__file__.rsplit("/", 1)[0]}/{name}.npz'))


def b200(c, gross=None, frames=None):
    cor = framecor.Correlator(c['height'], c['width'], c['down'], c['across'], window=c['window'],
                              search=c['search'], stat_size=c['stat_size'], backend='b200')
    cor.set_reference(c['reference'])
    return cor, cor.correlate(c['frames'] if frames is None else frames, gross=c['gross'] if gross is None else gross)


def subgrid(name):
    """the frames, rows and columns of windows a case is checked on against the FP64 oracle"""
    a, b = cases.SUBGRID.get(name, (1, 1))
    return (slice(None), slice(None, None, a), slice(None, None, b))


def sub(c, sl):
    """The windows and the gross offsets of the sub-grid sl (frames, rows, columns) of case c."""
    g = oracle.expand_gross(c['gross'], len(c['frames']), len(c['down']), len(c['across']))
    return c['down'][sl[1]], c['across'][sl[2]], None if g is None else g[sl]


def fp64_surface(c, down, across, gross, f, y, x):
    g = None if gross is None else gross[f:f + 1, y:y + 1, x:x + 1]
    o = oracle.correlate(c['height'], c['width'], down[y:y + 1], across[x:x + 1], c['reference'],
                         c['frames'][f:f + 1], g, window=c['window'], search=c['search'],
                         stat_size=c['stat_size'], mode='f64', surfaces=True)
    return o['surface'][0, 0, 0], (0, 0) if g is None else tuple(g[0, 0, 0])


def near_tie_ok(c, mism, out, ref_out, tol, sl=(slice(None),) * 3):
    """Mismatched integer peaks are near-ties: on the oracle's FP64 surface the value at each
    side's peak shift is within tol of the maximum (out and ref_out on the sub-grid sl)."""
    if not mism.any():
        return True
    down, across, gross = sub(c, sl)
    R, M = c['search'], 2 * c['search'] + 1
    for ff, yy, xx in np.argwhere(mism):
        s, (gy, gx) = fp64_surface(c, down, across, gross, ff, yy, xx)
        for res in (out, ref_out):
            u = int(np.rint(res['offsets'][ff, yy, xx, 0] - gy + R))
            v = int(np.rint(res['offsets'][ff, yy, xx, 1] - gx + R))
            cand = s[max(u - 1, 0):min(u + 2, M), max(v - 1, 0):min(v + 2, M)].max()
            if s.max() - cand > tol:
                return False
    return True


def default_is_tc(c, cor):
    """whether the library's default form for case c is the tensor-core form: windows above 32 px at
    FFT sizes up to 160 and searches up to 63 px"""
    return c['window'] > 32 and cor.info()[2] <= 160 and c['search'] <= 63


def tie_count(c, tol=NEAR_TIE, sl=(slice(None),) * 3):
    """The pairs whose FP64 surface holds another shift within tol of its maximum: the only pairs
    whose integer peak rounding may decide. 'mixed' (flat, saturated and 8 px striped regions) has
    182 of 456 (exact ties); the other small cases have none."""
    down, across, gross = sub(c, sl)
    o = oracle.correlate(c['height'], c['width'], down, across, c['reference'], c['frames'], gross,
                         window=c['window'], search=c['search'], stat_size=c['stat_size'], mode='f64', surfaces=True)
    M = 2 * c['search'] + 1
    flat = o['surface'].reshape(-1, M * M)
    valid = np.isfinite(o['offsets'][..., 0]).reshape(-1)
    n = 0
    for p in np.flatnonzero(valid):
        f = flat[p].copy()
        top = f.max()
        f[int(np.argmax(f))] = -np.inf
        n += int(top - f.max() <= tol)
    return n


@pytest.mark.parametrize('name', SUPPORTED)
def test_golden(name):
    """b200 against the reference CPU backend's outputs."""
    c, g = cases.case(name), golden(name)
    assert str(g['digest']) == cases.digest(c)
    cor, r = b200(c)
    a, b = g['offsets'], r['offsets']
    assert np.array_equal(np.isnan(a), np.isnan(b))
    valid = np.isfinite(a[..., 0])
    assert np.all(r['snr'][~valid] == 0) and np.all(r['peak'][~valid] == 0)
    assert np.all(r['cov'][~valid] == np.array([99, 99, 0], np.float32))
    d = np.abs(a - b).max(-1)
    mism = valid & (d > 0.1)
    if mism.any():   # every differing peak is a verified near-tie of the form that ran (the default)
        tol = TC_NEAR_TIE if default_is_tc(c, cor) else NEAR_TIE
        assert near_tie_ok(c, mism, r, g, tol), f'{mism.sum()} peaks differ'
    ok = valid & ~mism
    assert d[ok].max() < 1e-3, d[ok].max()
    assert np.abs(g['peak'][ok] - r['peak'][ok]).max() < 1e-4
    assert np.abs(r['snr'][ok] / g['snr'][ok] - 1).max() < 1e-2


@pytest.mark.parametrize('name', ['shifts', 'gross', 'window_gross', 'small', 'hd', 'wide', 'mixed', *cases.C3])
def test_fp64_oracle(name):
    """b200 against the FP64 direct-correlation oracle: the 0.01 px gate."""
    c = cases.case(name)
    cor, r = b200(c)
    sl = subgrid(name)
    down, across, gross = c['down'][sl[1]], c['across'][sl[2]], c['gross']
    o = oracle.correlate(c['height'], c['width'], down, across, c['reference'], c['frames'],
                         gross if gross is None or gross.ndim == 2 else gross[sl], window=c['window'],
                         search=c['search'], stat_size=c['stat_size'], mode='f64')
    b = {k: v[sl] for k, v in r.items()}
    assert np.array_equal(np.isnan(o['offsets']), np.isnan(b['offsets']))
    valid = np.isfinite(o['offsets'][..., 0])
    d = np.abs(o['offsets64'] - b['offsets']).max(-1)
    mism = valid & (d > 0.1)
    if mism.any():   # per-frame and per-window gross alike; near-ties of the form that ran
        tol = TC_NEAR_TIE if default_is_tc(c, cor) else NEAR_TIE
        assert mism.sum() <= tie_count(c, tol, sl)
        assert near_tie_ok(c, mism, b, o, tol, sl)
    ok = valid & ~mism
    assert d[ok].max() < 0.01, d[ok].max()
    assert np.abs(b['snr'][ok] / o['snr'][ok] - 1).max() < 1e-3
    assert np.abs(b['peak'][ok] - o['peak'][ok]).max() < 1e-5


def test_surfaces():
    """The normalized surfaces against the oracle's float restatement."""
    c = cases.case('shifts')
    cor = framecor.Correlator(c['height'], c['width'], c['down'], c['across'], window=c['window'],
                              search=c['search'], backend='b200')
    cor.set_reference(c['reference'])
    r = cor.correlate(torch.as_tensor(c['frames']).cuda(), surfaces=True)
    s = r['surface'].cpu().numpy()
    o = oracle.correlate(c['height'], c['width'], c['down'], c['across'], c['reference'], c['frames'],
                         window=c['window'], search=c['search'], mode='ref32', surfaces=True)
    assert np.abs(s - o['surface']).max() < 2e-5


@pytest.mark.parametrize('shape', [(720, 1280), (37, 53), (1, 1), (300, 129), (64, 4096)])
def test_sat_bitexact(shape):
    rng = np.random.default_rng(shape[0] * 7 + shape[1])
    f = rng.integers(0, 256, (3,) + shape, dtype=np.uint8)
    f[1] = 255
    s32, s64 = framecor.sat(torch.as_tensor(f).cuda())
    for k in range(3):
        a, a2 = oracle.sat(f[k])
        assert np.array_equal(s32[k].cpu().numpy(), a & 0xFFFFFFFF)
        assert np.array_equal(s64[k].cpu().numpy(), a2)


def test_sat_wraps_exactly():
    """A frame whose pixel sum passes 2^32: the 32-bit table is the exact one modulo 2^32."""
    f = np.full((1, 4096, 4500), 255, np.uint8)
    s32, s64 = framecor.sat(torch.as_tensor(f).cuda())
    a, a2 = oracle.sat(f[0])
    assert a[-1, -1] > 2 ** 32
    assert np.array_equal(s32[0].cpu().numpy(), a & 0xFFFFFFFF)
    assert np.array_equal(s64[0].cpu().numpy(), a2)


def test_gross_broadcast_bitexact():
    c = cases.case('hd')
    cor, r1 = b200(c)
    g = np.ascontiguousarray(np.broadcast_to(c['gross'][:, None, None, :], (2,) + cor.shape + (2,)))
    r2 = cor.correlate(c['frames'], gross=g)
    for k in r1:
        assert np.array_equal(r1[k], r2[k], equal_nan=True), k


def test_device_equals_host():
    c = cases.case('window_gross')
    cor, r1 = b200(c)
    r2 = cor.correlate(torch.as_tensor(c['frames']).cuda(), gross=torch.as_tensor(c['gross']).cuda())
    for k in r1:
        assert np.array_equal(r1[k], r2[k].cpu().numpy(), equal_nan=True), k


@pytest.mark.parametrize('form', ['tc', 'int8'])
@pytest.mark.parametrize('pad', [4, 5])
def test_rows_off_16_byte_boundaries_give_the_same_outputs(form, pad):
    """The tensor-core forms read frames whose rows start on 16-byte boundaries with 16-byte chunks
    (the gather, the refinement's staging) and other frames with 4-byte words or bytes: the same
    frames, in rows pad bytes off those boundaries (the device entry point with a pitch; the Python
    device path would make them contiguous), give identical outputs, with per-window gross offsets
    moving the chips to every byte alignment."""
    from slipcam_b200 import _lib
    h, w = 360, 640
    frames = synth.video(h, w, 4, np.array([[0.0, 0.0], [1.4, -2.6], [-3.1, 0.8], [2.2, 2.9]]), np.zeros(4),
                         sigma=1.5, noise=1.5, seed=21 + pad)
    down, across = framecor.window_grid(h, w, 64, 48, 16)
    cor = framecor.Correlator(h, w, down, across, window=64, search=48, backend='b200')
    cor.set_form(form)
    cor.set_reference(frames[0])
    rng = np.random.default_rng(3 + pad)
    gross = torch.as_tensor(rng.integers(-9, 10, (3, len(down), len(across), 2)).astype(np.int32)).cuda()
    t = torch.as_tensor(frames[1:]).cuda()
    big = torch.zeros((3, h, w + pad), dtype=torch.uint8, device='cuda')
    big[:, :, pad:] = t

    def run(ptr, pitch):
        ny, nx = cor.shape
        out = [torch.empty((3, ny, nx, 2), dtype=torch.float32, device='cuda'),
               torch.empty((3, ny, nx), dtype=torch.float32, device='cuda'),
               torch.empty((3, ny, nx), dtype=torch.float32, device='cuda'),
               torch.empty((3, ny, nx, 3), dtype=torch.float32, device='cuda')]
        rc = _lib.lib().b200_correlate_device(cor._h, ptr, 3, pitch, gross.data_ptr(), _lib.GROSS_WINDOW,
                                              *[o.data_ptr() for o in out], torch.cuda.current_stream().cuda_stream)
        _lib.raise_for(rc, cor._h)
        return out

    aligned = run(t.data_ptr(), w)
    off = run(big.data_ptr() + pad, w + pad)
    for x, y in zip(aligned, off):
        assert torch.equal(torch.nan_to_num(x, 7.0), torch.nan_to_num(y, 7.0))
    assert torch.isfinite(aligned[0]).float().mean() > 0.9
    cor.check()


def test_many_groups_host_path():
    """More frames than one launch group: the double-buffered host path keeps every frame's
    outputs in place (the same frames correlated one call at a time agree exactly)."""
    frames, motion, step = synth.small(n=40, h=180, w=320)
    down, across = framecor.window_grid(180, 320, 32, 16, 16)
    cor = framecor.Correlator(180, 320, down, across, window=32, search=16, backend='b200')
    cor.set_reference(frames[0])
    all_at_once = cor.correlate(frames)
    for k in (0, 17, 39):
        one = cor.correlate(frames[k:k + 1])
        for key in one:
            assert np.array_equal(one[key][0], all_at_once[key][k], equal_nan=True), (k, key)


def test_hd_recovers_motion():
    """720p, window 64, search 48 (the headline geometry), a full frame grid: the offsets of the
    windows on the near side of the fault are the camera motion."""
    frames, motion, step, gross = synth.hd(n=3, device='cuda')
    down, across = framecor.window_grid(720, 1280, 64, 48, 16)
    cor = framecor.Correlator(720, 1280, down, across, window=64, search=48, backend='b200')
    cor.set_reference(frames[0])
    r = cor.correlate(frames[1:], gross=torch.as_tensor(gross[1:]).cuda())
    off = r['offsets'].cpu().numpy()
    for k in range(2):
        err = off[k] - motion[k + 1][None, None, :]
        assert np.nanmedian(np.abs(err)) < 0.05


# ---- the tensor-core form (FP16 operands, FP32 accumulation), its peaks refined exactly: the 3 x 3
# values around each integer peak are recomputed in integers (tc_refine_kernel), so the offsets,
# the peak value and the covariance are the exact form's; the SNR keeps the FP16 values of the rest
# of its patch. The gates are the FP32 form's, on every case: offsets within 0.01 px, SNR within
# 1e-3 relative of the FP64 oracle, integer peaks identical except near-ties of the FP16 surface.
TC_CASES = ['shifts', 'gross', 'window_gross', 'invalid', 'small', 'hd', 'mixed', 'c3_w32', 'c3_w64']


@pytest.mark.parametrize('name', TC_CASES)
def test_tc_fp64_oracle(name):
    c = cases.case(name)
    cor = framecor.Correlator(c['height'], c['width'], c['down'], c['across'], window=c['window'],
                              search=c['search'], stat_size=c['stat_size'], backend='b200')
    cor.set_form('tc')
    cor.set_reference(c['reference'])
    r = cor.correlate(c['frames'], gross=c['gross'])
    sl = subgrid(name)
    down, across, gross = c['down'][sl[1]], c['across'][sl[2]], c['gross']
    o = oracle.correlate(c['height'], c['width'], down, across, c['reference'], c['frames'],
                         gross if gross is None or gross.ndim == 2 else gross[sl], window=c['window'],
                         search=c['search'], stat_size=c['stat_size'], mode='f64')
    b = {k: v[sl] for k, v in r.items()}
    assert np.array_equal(np.isnan(o['offsets']), np.isnan(b['offsets']))
    valid = np.isfinite(o['offsets'][..., 0])
    assert np.all(b['cov'][~valid] == np.array([99, 99, 0], np.float32))
    d = np.abs(o['offsets64'] - b['offsets']).max(-1)
    mism = valid & (d > 0.1)
    if mism.any():   # each one a near-tie within the FP16 surface error
        assert mism.sum() <= tie_count(c, TC_NEAR_TIE, sl)
        assert near_tie_ok(c, mism, b, o, TC_NEAR_TIE, sl)
    ok = valid & ~mism
    assert np.abs(b['peak'][ok] - o['peak'][ok]).max() < 1e-6
    assert d[ok].max() < 0.01, d[ok].max()
    snr_rel = np.abs(b['snr'][ok] / o['snr'][ok] - 1)
    assert snr_rel.max() < 1e-3, snr_rel.max()


def test_tc_surfaces_close_to_fft32():
    c = cases.case('hd')
    cor = framecor.Correlator(c['height'], c['width'], c['down'], c['across'], window=64, search=48, backend='b200')
    cor.set_form('fft32')
    cor.set_reference(c['reference'])
    f = torch.as_tensor(c['frames']).cuda()
    g = torch.as_tensor(c['gross']).cuda()
    s32 = cor.correlate(f, gross=g, surfaces=True)['surface']
    cor.set_form('tc')
    stc = cor.correlate(f, gross=g, surfaces=True)['surface']
    assert torch.isfinite(stc).all()
    assert (stc - s32).abs().max().item() < 2e-3


def test_tc_form_limits():
    """Geometries the tensor-core kernel does not hold are refused with a ValueError."""
    down, across = framecor.window_grid(512, 512, 64, 64, 64)   # L = 192
    cor = framecor.Correlator(512, 512, down, across, window=64, search=64, backend='b200')
    with pytest.raises(ValueError, match='tensor-core'):
        cor.set_form('tc')
    with pytest.raises(ValueError):
        cor.set_form('bf16')


def test_big_transform_surfaces_match_fp64_oracle():
    """L = 256 (window 128, search 64): the staged N = 256 transform's surfaces against the FP64
    direct oracle on every pair of the golden case."""
    c = cases.case('big')
    cor = framecor.Correlator(c['height'], c['width'], c['down'], c['across'], window=128, search=64,
                              stat_size=c['stat_size'], backend='b200')
    cor.set_reference(c['reference'])
    assert cor.info()[2] == 256
    out = cor.correlate(torch.as_tensor(c['frames']).cuda(), surfaces=True)
    o = oracle.correlate(c['height'], c['width'], c['down'], c['across'], c['reference'], c['frames'], None,
                         window=128, search=64, stat_size=c['stat_size'], mode='f64', surfaces=True)
    assert np.abs(out['surface'].cpu().numpy() - o['surface']).max() < 2e-5
    d = np.abs(out['offsets'].cpu().numpy() - o['offsets64'])
    assert np.array_equal(np.isnan(d), np.isnan(o['offsets64']))
    assert np.nanmax(d) < 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize('window,search', [(127, 64), (130, 60), (200, 10)])
def test_big_transform_cluster_geometries(window, search):
    """The two-CTA cluster form of the N = 256 transform at other geometries than the golden case: odd
    L (the last chip row padded), other surface sizes (other splits of the M rows between the two
    CTAs), a small search. Surfaces and offsets against the FP64 direct oracle."""
    from slipcam_b200 import synth
    h, w = 360, 400
    frames = synth.video(h, w, 2, np.array([[0.0, 0.0], [1.3, -2.2]]), np.zeros(2), sigma=2.0, noise=1.0, seed=21)
    down, across = framecor.window_grid(h, w, window, search, 48)
    down, across = down[:2], across[:2]
    cor = framecor.Correlator(h, w, down, across, window=window, search=search, backend='b200')
    cor.set_reference(frames[0])
    assert cor.info()[2] == 256
    out = cor.correlate(torch.as_tensor(frames[1:]).cuda(), surfaces=True)
    o = oracle.correlate(h, w, down, across, frames[0], frames[1:], None, window=window, search=search, mode='f64',
                         surfaces=True)
    assert np.abs(out['surface'].cpu().numpy() - o['surface']).max() < 2e-5
    d = np.abs(out['offsets'].cpu().numpy() - o['offsets64'])
    assert np.array_equal(np.isnan(d), np.isnan(o['offsets64']))
    assert np.nanmax(d) < 1e-3


def test_search_beyond_big_transform_rejected():
    """Past the staged transform's limit (search 64 at L up to 256) a clear ValueError."""
    down, across = framecor.window_grid(512, 512, 32, 100, 64)   # L = 232, M = 201
    with pytest.raises(ValueError, match='searches up to 64'):
        framecor.Correlator(512, 512, down, across, window=32, search=100, backend='b200')
