"""
The C ABI library without a GPU: it loads, it exports every entry point include/slipcam_b200.h
declares, and the argument checks that come before any device work behave like the reference's
(cxx/common.cpp:15-28, bindings.cpp:38-44). CPU only.
"""

import os
import re

import pytest

from slipcam_b200 import _lib, framecor

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for f in os.listdir(os.path.join(ROOT, 'include')):
        if f.endswith('.h'):
            text = open(os.path.join(ROOT, 'include', f)).read()
            names |= set(re.findall(r'^B200_API\s+[\w\s\*]*?\b(b200_\w+)\s*\(', text, re.M))
    return names


def test_library_loads():
    lib = _lib.lib()
    assert lib.b200_version() == b'0.1.0'
    assert framecor.__version__ == '0.1.0'


def test_exports_every_declared_symbol():
    names = declared()
    assert len(names) >= 14
    lib = _lib.lib()
    for name in names:
        assert hasattr(lib, name), name
    assert names <= set(_lib.SIGNATURES), 'a declared entry point has no ctypes signature'


def test_window_grid():
    """window_grid as python/slipcam/framecor/__init__.py:18-32."""
    down, across = framecor.window_grid(720, 1280, 64, 48, 16)
    assert len(down) == 35 and len(across) == 70 and down[0] == 48 and across[-1] == 48 + 16 * 69
    down, across = framecor.window_grid(240, 320, 32, 24, 24)
    assert (len(down), len(across)) == (6, 10)
    with pytest.raises(ValueError):
        framecor.window_grid(100, 100, 64, 48, 16)


@pytest.mark.parametrize('kwargs, match', [
    (dict(down=[0], across=[300]), 'outside the frame'),
    (dict(down=[-1], across=[0]), 'outside the frame'),
    (dict(down=[], across=[0]), 'no windows'),
    (dict(down=[0], across=[0], window=2), 'at least 3'),
    (dict(down=[0], across=[0], search=0), 'half search range'),
    (dict(down=[0], across=[0], stat_size=2), 'SNR window'),
    (dict(down=[0], across=[0], batch=0), 'batch'),
    (dict(down=[0], across=[0], backend='gpu'), 'backend'),
    (dict(down=[0], across=[0], backend='cpu'), 'backend'),
])
def test_argument_errors(kwargs, match):
    kw = dict(window=32, search=8)
    kw.update(kwargs)
    down, across = kw.pop('down'), kw.pop('across')
    with pytest.raises(ValueError, match=match):
        framecor.Correlator(240, 320, down, across, **kw)


def test_last_error_of_create():
    p = _lib.Params(0, 0, 32, 8, 21, 4096, None, 0, None, 0)
    import ctypes
    h = ctypes.c_void_p()
    assert _lib.lib().b200_create(ctypes.byref(p), 0, ctypes.byref(h)) == _lib.EINVAL
    assert h.value is None
    assert _lib.lib().b200_last_error(None).startswith(b'framecor: ')


def test_no_device_is_an_error():
    if framecor.has_cuda():
        pytest.skip('a B200 is present')
    with pytest.raises(RuntimeError):
        framecor.Correlator(240, 320, [0], [0], window=32, search=8)


def test_sat_rejects_bad_arguments():
    assert _lib.lib().b200_sat_device(None, -1, 10, 10, 10, None, None, None) == _lib.EINVAL
    assert _lib.lib().b200_sat_device(None, 1, 10, 10, 9, None, None, None) == _lib.EINVAL

