"""
ctypes binding of libslipcam_b200.so (include/slipcam_b200.h). The library must have been built
(``python -m slipcam_b200.build``); there is no fallback: every call goes to the CUDA library.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libslipcam_b200.so')

OK, EINVAL, ERUNTIME, ETIMEOUT = 0, 1, 2, 3
GROSS_NONE, GROSS_FRAME, GROSS_WINDOW = 0, 1, 2
FORM_AUTO, FORM_FFT32, FORM_TC, FORM_I8 = 0, 1, 2, 3
COARSE_MAX_WINDOWS = 2048
PERCENTILE_SCRATCH = 16640   # bytes of device scratch of b200_percentile_f32_device


class Params(ctypes.Structure):
    """b200_params"""
    _fields_ = [('height', ctypes.c_int), ('width', ctypes.c_int), ('window', ctypes.c_int),
                ('search', ctypes.c_int), ('stat_size', ctypes.c_int), ('batch', ctypes.c_int),
                ('down', ctypes.POINTER(ctypes.c_int32)), ('ny', ctypes.c_int),
                ('across', ctypes.POINTER(ctypes.c_int32)), ('nx', ctypes.c_int)]


# every entry point of include/slipcam_b200.h: name -> (restype, argtypes)
_vp, _i, _u8p = ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p
SIGNATURES = {
    'b200_create': (_i, [ctypes.POINTER(Params), _i, ctypes.POINTER(_vp)]),
    'b200_destroy': (_i, [_vp]),
    'b200_last_error': (ctypes.c_char_p, [_vp]),
    'b200_set_reference': (_i, [_vp, _u8p]),
    'b200_correlate': (_i, [_vp, _u8p, _i, _vp, _i, _vp, _vp, _vp, _vp]),
    'b200_set_reference_device': (_i, [_vp, _u8p, _i, _vp]),
    'b200_correlate_device': (_i, [_vp, _u8p, _i, _i, _vp, _i, _vp, _vp, _vp, _vp, _vp]),
    'b200_correlate_device_surfaces': (_i, [_vp, _u8p, _i, _i, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    'b200_correlate_device_noalloc': (_i, [_vp, _u8p, _i, _i, _vp, _i, _vp, _vp, _vp, _vp, _vp]),
    'b200_group_create': (_i, [ctypes.POINTER(_vp), _i, ctypes.POINTER(_vp)]),
    'b200_group_destroy': (_i, [_vp]),
    'b200_group_last_error': (ctypes.c_char_p, [_vp]),
    'b200_group_correlate_device': (_i, [_vp, _u8p, _i, _i, ctypes.POINTER(_vp), ctypes.POINTER(_i),
                                         ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                         ctypes.POINTER(_vp), _vp]),
    'b200_group_tune': (_i, [_vp, _u8p, _i, _i, ctypes.POINTER(_vp), ctypes.POINTER(_i), _vp,
                             ctypes.POINTER(ctypes.c_double)]),
    'b200_group_config': (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i),
                               ctypes.POINTER(_i)]),
    'b200_group_set_config': (_i, [_vp, _i, _i, _i, _i, _i]),
    'b200_periodicity_device': (_i, [_vp, _vp, _i, _vp, _vp]),
    'b200_ncc_peaks_device': (_i, [_vp, _i, _i, _vp, _vp]),
    'b200_stab_create': (_i, [_i, _i, _vp, _i, _i, ctypes.POINTER(_vp)]),
    'b200_stab_destroy': (_i, [_vp]),
    'b200_stab_last_error': (ctypes.c_char_p, [_vp]),
    'b200_stab_frames_device': (_i, [_vp, _vp, _i, _i, _vp, _vp, _vp, _vp]),
    'b200_warp_f32_device': (_i, [_vp, _i, _i, _vp, ctypes.c_float, _vp, _vp]),
    'b200_coarse_track_device': (_i, [_vp, _vp, _i, _i, _vp, ctypes.c_double, _i, _vp, _vp, _vp, _vp, _vp]),
    'b200_coarse_fit_device': (_i, [_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _i, ctypes.c_double, _vp, _vp, _vp,
                                    _vp]),
    'b200_frame_diff_device': (_i, [_vp, _i, _i, _i, _i, _vp, _vp, _vp]),
    'b200_chunk_std_median_device': (_i, [_vp, _i, _i, _i, _i, _i, _vp, _vp]),
    'b200_sobel_device': (_i, [_vp, _i, _i, _i, _vp, _vp]),
    'b200_percentile_f32_device': (_i, [_vp, ctypes.c_int64, ctypes.c_double, _vp, _vp, _vp]),
    'b200_text_mask_scratch_bytes': (ctypes.c_size_t, [_i, _i]),
    'b200_text_mask_device': (_i, [_vp, _vp, _i, _i, ctypes.c_double, ctypes.c_float, _i, _vp, _vp, ctypes.c_size_t,
                                   _vp]),
    'b200_set_reference_f32_device': (_i, [_vp, _vp, _i, _vp]),
    'b200_diff_forward': (_i, [_vp, _vp, _i, _i, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    'b200_diff_backward': (_i, [_vp, _vp, _i, _i, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    'b200_offset_adjoint': (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp]),
    'b200_sat_device': (_i, [_u8p, _i, _i, _i, _i, _vp, _vp, _vp]),
    'b200_set_form': (_i, [_vp, _i]),
    'b200_tc_selftest': (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _vp]),
    'b200_tc_i8_selftest': (_i, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _vp]),
    'b200_status': (_i, [_vp, _vp, ctypes.POINTER(ctypes.c_int)]),
    'b200_inject_alloc_failure': (_i, [_i]),
    'b200_host_copy': (_i, [_vp, _vp, ctypes.c_size_t]),
    'b200_wait_selftest': (_i, [ctypes.c_uint, ctypes.c_double, _vp]),
    'b200_info': (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i),
                       ctypes.POINTER(ctypes.c_uint64)]),
    'b200_profile': (_i, [_vp, _i]),
    'b200_profile_read': (_i, [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint64),
                               ctypes.POINTER(ctypes.c_uint64)]),
    'b200_backend': (ctypes.c_char_p, [_vp]),
    'b200_has_device': (_i, []),
    'b200_version': (ctypes.c_char_p, []),
}

_lib = None


def lib():
    """The loaded library; RuntimeError if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f'framecor: the b200 CUDA library is not built ({LIB_PATH}); '
                               'run python -m slipcam_b200.build')
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def loaded():
    """Whether the library can be loaded (without raising)."""
    try:
        lib()
        return True
    except (RuntimeError, OSError):
        return False


def raise_for(rc, handle=None, group=False):
    """The reference's exception for a status code (ValueError / RuntimeError)."""
    if rc == OK:
        return
    err = lib().b200_group_last_error if group else lib().b200_last_error
    msg = err(handle).decode() or f'framecor: error {rc}'
    if rc == EINVAL:
        raise ValueError(msg)
    raise RuntimeError(msg)
