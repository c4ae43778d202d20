"""
The oracle pinned against the reference: the C restatement (oracle/framecor_oracle.c), in both
modes, against the outputs of the reference's own CPU backend stored in tests/golden (CPU only).
"""

import numpy as np
import pytest

import cases

SUBGRID = cases.SUBGRID   # the oracle sums directly: a sub-grid of the 720p windows


def load(name):
    c = cases.case(name)
    g = dict(np.load(f'{cases.__file__.rsplit("/", 1)[0]}/{name}.npz'))
    return c, g


def sub(c, g, name):
    down, across = c['down'], c['across']
    gross = c['gross']
    if name in SUBGRID:
        a, b = SUBGRID[name]
        down, across = down[::a], across[::b]
        g = {k: (v[:, ::a, ::b] if k != 'digest' else v) for k, v in g.items()}
        if gross is not None and gross.ndim == 4:
            gross = gross[:, ::a, ::b]
    return down, across, gross, g


@pytest.mark.parametrize('name', cases.NAMES)
def test_golden_inputs(name):
    """The inputs regenerate bit for bit (the fixtures were made from these)."""
    c, g = load(name)
    assert str(g['digest']) == cases.digest(c)


def compare(ref, out, *, off_tol, peak_tol, snr_rtol):
    """The reference's outputs vs ours: the same invalid pairs (NaN offsets, zero SNR and peak,
    cov (99, 99, 0)); the valid ones within the tolerances."""
    a, b = ref['offsets'], out['offsets']
    assert np.array_equal(np.isnan(a), np.isnan(b))
    valid = np.isfinite(a[..., 0])
    assert np.all(ref['snr'][~valid] == 0) and np.all(out['snr'][~valid] == 0)
    assert np.all(out['peak'][~valid] == 0)
    assert np.all(out['cov'][~valid] == np.array([99, 99, 0], np.float32))
    if valid.any():
        assert np.abs(a[valid] - b[valid]).max() < off_tol
        assert np.abs(ref['peak'][valid] - out['peak'][valid]).max() < peak_tol
        assert np.abs(out['snr'][valid] / ref['snr'][valid] - 1).max() < snr_rtol


@pytest.mark.parametrize('mode', ['ref32', 'f64'])
@pytest.mark.parametrize('name', cases.NAMES)
def test_oracle_vs_reference(oracle_mod, name, mode):
    """Both oracle modes reproduce the reference CPU backend: offsets within 1e-4 px (the
    reference's FFT rounding), peak within 1e-6, SNR within 1e-5 relative."""
    c, g = load(name)
    down, across, gross, g = sub(c, g, name)
    o = oracle_mod.correlate(c['height'], c['width'], down, across, c['reference'], c['frames'], gross,
                             window=c['window'], search=c['search'], stat_size=c['stat_size'], mode=mode)
    compare(g, o, off_tol=1e-4, peak_tol=1e-6, snr_rtol=1e-5)


def test_sat(oracle_mod):
    """The oracle's summed-area tables are numpy's cumulative sums."""
    rng = np.random.default_rng(0)
    f = rng.integers(0, 256, (37, 53), dtype=np.uint8)
    s, s2 = oracle_mod.sat(f)
    ref = np.zeros((38, 54), np.int64)
    ref[1:, 1:] = f.astype(np.int64).cumsum(0).cumsum(1)
    ref2 = np.zeros((38, 54), np.int64)
    ref2[1:, 1:] = (f.astype(np.int64) ** 2).cumsum(0).cumsum(1)
    assert np.array_equal(s, ref) and np.array_equal(s2, ref2)


def test_reference_windows(oracle_mod):
    """Zero-mean windows and their norms (cxx/common.cpp:30-48)."""
    c = cases.case('shifts')
    win, norms = oracle_mod.reference_windows(c['height'], c['width'], c['down'], c['across'], c['window'],
                                              c['reference'])
    W = c['window']
    y0, x0 = c['down'][1], c['across'][2]
    k = 1 * len(c['across']) + 2
    patch = c['reference'][y0:y0 + W, x0:x0 + W].astype(np.float64)
    assert np.allclose(win[k], patch - patch.mean(), atol=1e-4)
    assert abs(norms[k] - np.sqrt(((patch - patch.mean()) ** 2).sum())) < 1e-3


def test_oracle_recovers_shifts(oracle_mod):
    """The reference test's known-shift recovery, on the oracle."""
    c = cases.case('shifts')
    o = oracle_mod.correlate(c['height'], c['width'], c['down'], c['across'], c['reference'], c['frames'],
                             window=c['window'], search=c['search'], mode='f64')
    for k, s in enumerate([(0, 0), (0.3, -0.7), (5.25, -12.5), (-20.4, 15.1)]):
        err = o['offsets'][k] - np.array(s, np.float32)
        assert np.median(np.abs(err)) < 0.05 and np.abs(err).max() < 0.25
