"""NIFTY-style interface (reference python/curagridder/cursl.py:78-166).

``ms2dirty(uvw, freq, ms, wgt, nxdirty, nydirty, rad_pix_x, rad_pix_y, nx, ny,
epsilon, do_wstacking, *args)`` returns the real dirty image; ``dirty2ms(uvw,
freq, dirty, wgt, rad_pix_x, rad_pix_y, nx, ny, epsilon, do_wstacking, *args)``
returns visibilities of shape (nrow, 1).  As in the reference: sign = -1,
sigma = 2, fov = rad_pix_x * nxdirty in degrees (both axes), only freq[0] is
used, complex128 visibilities select the FP64 path and complex64 the FP32 path.
"""
import numpy as np

from . import _lib
from .curagridder import (dirty2ms_1, dirty2ms_2, dirty2msf_1, dirty2msf_2, ms2dirty_1,
                          ms2dirty_2, ms2dirtyf_1, ms2dirtyf_2)


def _flat(a, dtype):
    return np.ascontiguousarray(np.asarray(a).reshape(-1), dtype=dtype)


def ms2dirty(uvw, freq, ms, wgt, nxdirty, nydirty, rad_pix_x, rad_pix_y, nx, ny, epsilon,
             do_wstacking, *args):
    """Dirty image [nxdirty, nydirty] (real part) from visibilities ``ms``."""
    nrow = uvw.shape[0]
    sigma = 2
    fov = rad_pix_x * nxdirty * 180 / np.pi
    sign = -1
    single = np.asarray(ms).dtype != np.complex128
    if single:
        dirty = np.zeros((nxdirty, nydirty), dtype=np.complex64)
        u = np.ascontiguousarray(uvw, dtype=np.float32)
        m = _flat(ms, np.complex64)
        if wgt is None:
            r = ms2dirtyf_1(nrow, nxdirty, nydirty, fov, freq[0], u, m, dirty, epsilon, sigma, sign)
        else:
            r = ms2dirtyf_2(nrow, nxdirty, nydirty, fov, freq[0], u, m, _flat(wgt, np.float32),
                            dirty, epsilon, sigma, sign)
    else:
        dirty = np.zeros((nxdirty, nydirty), dtype=np.complex128)
        u = np.ascontiguousarray(uvw, dtype=np.float64)
        m = _flat(ms, np.complex128)
        if wgt is None:
            r = ms2dirty_1(nrow, nxdirty, nydirty, fov, freq[0], u, m, dirty, epsilon, sigma, sign)
        else:
            r = ms2dirty_2(nrow, nxdirty, nydirty, fov, freq[0], u, m, _flat(wgt, np.float64),
                           dirty, epsilon, sigma, sign)
    _lib.check(r)
    return dirty.real


def dirty2ms(uvw, freq, dirty, wgt, rad_pix_x, rad_pix_y, nx, ny, epsilon, do_wstacking, *args):
    """Visibilities (nrow, 1) from a real dirty image [nxdirty, nydirty]."""
    nrow = uvw.shape[0]
    nxdirty, nydirty = dirty.shape[0], dirty.shape[1]
    sigma = 2
    fov = rad_pix_x * nxdirty * 180 / np.pi
    sign = -1
    if dirty.dtype == np.float64:
        u = np.ascontiguousarray(uvw, dtype=np.float64)
        ms = np.zeros((nrow, 1), dtype=np.complex128)
        dirty1 = np.zeros(dirty.shape, dtype=np.complex128)
    else:
        u = np.ascontiguousarray(uvw, dtype=np.float32)
        ms = np.zeros((nrow, 1), dtype=np.complex64)
        dirty1 = np.zeros(dirty.shape, dtype=np.complex64)
    dirty1.real = dirty
    if wgt is None:
        fn = dirty2ms_1 if dirty.dtype == np.float64 else dirty2msf_1
        r = fn(nrow, nxdirty, nydirty, fov, freq[0], u, ms, dirty1, epsilon, sigma, sign)
    else:
        fn, wt = (dirty2ms_2, np.float64) if dirty.dtype == np.float64 else (dirty2msf_2, np.float32)
        r = fn(nrow, nxdirty, nydirty, fov, freq[0], u, ms, _flat(wgt, wt), dirty1, epsilon, sigma,
               sign)
    _lib.check(r)
    return ms
