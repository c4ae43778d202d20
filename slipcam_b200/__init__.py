"""
slipcam_b200: slipcam framecor's correlator (Correlator.correlate, the dense normalized
cross-correlation of uint8 video frames with a reference frame) as a B200-native backend.

    from slipcam_b200 import framecor
    cor = framecor.Correlator(h, w, *framecor.window_grid(h, w, 64, 48, 16), backend='b200')

The compute is hand-written sm_100a CUDA in libslipcam_b200.so (include/slipcam_b200.h).
"""

__version__ = '0.1.0'
