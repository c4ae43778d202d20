"""
Generate tests/golden/<case>.npz: the outputs of the reference's own CPU backend (slipcam
cxx/cpu.cpp + cxx/common.cpp + cxx/bindings.cpp, compiled unchanged by oracle/Makefile against the
project's FFTW-API shim) on the seeded inputs of tests/golden/cases.py.

Each file holds offsets, peak, snr, cov (float32, the reference's dict) and 'digest', the sha256
of the inputs they were computed from (tests regenerate the inputs and check it).

usage: python tests/golden/make_golden.py [case ...]    (needs the reference sources to build)
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import cases  # noqa: E402
from oracle import oracle  # noqa: E402


def main(names):
    oracle.build()
    ref = oracle.reference_module()
    if ref is None:
        raise SystemExit('the reference module is not built (oracle/_ref)')
    for name in names:
        c = cases.case(name)
        cor = ref.Correlator(c['height'], c['width'], list(c['down']), list(c['across']), window=c['window'],
                             search=c['search'], backend='cpu', stat_size=c['stat_size'])
        cor.set_reference(c['reference'])
        r = cor.correlate(c['frames'], gross=c['gross'])
        out = {k: np.asarray(r[k]) for k in ('offsets', 'peak', 'snr', 'cov')}
        np.savez_compressed(os.path.join(HERE, f'{name}.npz'), digest=cases.digest(c), **out)
        valid = np.isfinite(out['offsets'][..., 0]).mean()
        print(f'{name}: {out["peak"].size} pairs, {valid:.0%} valid, median snr {np.median(out["snr"]):.1f}')


if __name__ == '__main__':
    main(sys.argv[1:] or cases.NAMES)
