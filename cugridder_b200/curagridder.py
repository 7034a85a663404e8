"""ctypes binding with the reference's names and argument order.

Mirrors python/curagridder/curagridder.py of the reference: module-level
``ms2dirty_1/_2``, ``dirty2ms_1/_2`` (FP64) and ``ms2dirtyf_*``/``dirty2msf_*``
(FP32) callables taking numpy arrays, and ``vis2dirty`` / ``dirty2vis``
(sign = +1, reference curagridder.py:92-151).  The numpy argument checks of the
reference's ``ndpointer`` argtypes (C-contiguous, exact dtype) are kept.  One
deliberate difference: the reference declares ``ms2dirtyf_2``'s fov and freq as
c_double (curagridder.py:77); here every FP32 entry point takes c_float, which
is what the C function expects.
"""
import numpy as np

from . import _lib


def _arr(a, dtype, name):
    if not isinstance(a, np.ndarray):
        raise TypeError("%s: expected a numpy array" % name)
    if a.dtype != dtype:
        raise TypeError("%s: array must have data type %s" % (name, np.dtype(dtype)))
    if not a.flags["C_CONTIGUOUS"]:
        raise TypeError("%s: array must be C-contiguous" % name)
    return a.ctypes.data


def _make(name, real, cplx, has_wgt):
    def call(nrow, nxdirty, nydirty, fov, freq, uvw, ms, *rest):
        fn = getattr(_lib.load(), name)
        if has_wgt:
            wgt, dirty, epsilon, sigma, sign = rest
        else:
            dirty, epsilon, sigma, sign = rest
            wgt = None
        args = [int(nrow), int(nxdirty), int(nydirty), fov, freq, _arr(uvw, real, "uvw"),
                _arr(ms, cplx, "ms")]
        if has_wgt:
            args.append(_arr(wgt, real, "wgt"))
        args += [_arr(dirty, cplx, "dirty"), epsilon, sigma, int(sign)]
        return fn(*args)

    call.__name__ = name
    call.__doc__ = "libcugridder %s (reference cugridder.h signature); returns the status code." % name
    return call


ms2dirty_1 = _make("ms2dirty_1", np.float64, np.complex128, False)
ms2dirty_2 = _make("ms2dirty_2", np.float64, np.complex128, True)
dirty2ms_1 = _make("dirty2ms_1", np.float64, np.complex128, False)
dirty2ms_2 = _make("dirty2ms_2", np.float64, np.complex128, True)
ms2dirtyf_1 = _make("ms2dirtyf_1", np.float32, np.complex64, False)
ms2dirtyf_2 = _make("ms2dirtyf_2", np.float32, np.complex64, True)
dirty2msf_1 = _make("dirty2msf_1", np.float32, np.complex64, False)
dirty2msf_2 = _make("dirty2msf_2", np.float32, np.complex64, True)


def vis2dirty(uvw, freq, ms, wgt, dirty, fov, epsilon=1e-6, sigma=2):
    """Image from visibilities (sign = +1), written into ``dirty`` [nx, ny] complex128.

    Reference: python/curagridder/curagridder.py:92-121.
    """
    nrow = uvw.shape[0]
    nxdirty, nydirty = dirty.shape[0], dirty.shape[1]
    sign = 1
    if wgt is None:
        r = ms2dirty_1(nrow, nxdirty, nydirty, fov, freq[0], uvw, ms, dirty, epsilon, sigma, sign)
    else:
        r = ms2dirty_2(nrow, nxdirty, nydirty, fov, freq[0], uvw, ms, wgt, dirty, epsilon, sigma,
                       sign)
    _lib.check(r)
    return dirty


def dirty2vis(uvw, freq, ms, wgt, dirty, fov, epsilon=1e-6, sigma=2):
    """Visibilities from an image (sign = +1), written into ``ms`` complex128.

    Reference: python/curagridder/curagridder.py:123-151.
    """
    nrow = uvw.shape[0]
    nxdirty, nydirty = dirty.shape[0], dirty.shape[1]
    sign = 1
    if wgt is None:
        r = dirty2ms_1(nrow, nxdirty, nydirty, fov, freq[0], uvw, ms, dirty, epsilon, sigma, sign)
    else:
        r = dirty2ms_2(nrow, nxdirty, nydirty, fov, freq[0], uvw, ms, wgt, dirty, epsilon, sigma,
                       sign)
    _lib.check(r)
    return ms
