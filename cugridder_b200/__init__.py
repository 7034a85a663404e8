"""cugridder_b200: B200-native (sm_100a) radio-interferometric gridder.

Drop-in for the ms2dirty / dirty2ms path of RapidsAtHKUST/cuGridder:

* ``libcugridder.so`` exports the reference's C ABI (``ms2dirty_1/_2``,
  ``dirty2ms_1/_2`` and the FP32 ``ms2dirtyf_*``/``dirty2msf_*``) plus a
  precision-split host API and a device-pointer plan API (include/cugridder.h);
* this package mirrors the reference's ``curig`` ctypes binding
  (``ms2dirty``/``dirty2ms`` NIFTY-style, ``vis2dirty``/``dirty2vis``) and adds
  :class:`Plan` for device-resident data.
"""
from . import _lib
from ._lib import GridderError
from .curagridder import (dirty2ms_1, dirty2ms_2, dirty2msf_1, dirty2msf_2, dirty2vis,
                          ms2dirty_1, ms2dirty_2, ms2dirtyf_1, ms2dirtyf_2, vis2dirty)
from .cursl import dirty2ms, ms2dirty
from .plan import Plan

__all__ = [
    "ms2dirty", "dirty2ms", "vis2dirty", "dirty2vis", "Plan", "GridderError",
    "ms2dirty_1", "ms2dirty_2", "dirty2ms_1", "dirty2ms_2",
    "ms2dirtyf_1", "ms2dirtyf_2", "dirty2msf_1", "dirty2msf_2",
    "ms2dirty_mixed", "dirty2ms_mixed", "release_cache", "set_host_kernel",
]


def ms2dirty_mixed(uvw, freq, vis, wgt, nxdirty, nydirty, fov_deg, epsilon, sigma=2.0, sign=-1):
    """Precision-split ms2dirty on HOST arrays: uvw float64, vis complex64,
    wgt float32 (or None); returns the complex64 dirty image [nx, ny]."""
    import numpy as np

    uvw = np.ascontiguousarray(uvw, dtype=np.float64)
    vis = np.ascontiguousarray(np.asarray(vis).reshape(-1), dtype=np.complex64)
    w = None if wgt is None else np.ascontiguousarray(np.asarray(wgt).reshape(-1), dtype=np.float32)
    dirty = np.zeros((nxdirty, nydirty), dtype=np.complex64)
    r = _lib.load().cg_ms2dirty_mixed(uvw.shape[0], nxdirty, nydirty, fov_deg, freq, uvw.ctypes.data,
                                      vis.ctypes.data, None if w is None else w.ctypes.data,
                                      dirty.ctypes.data, epsilon, sigma, sign)
    _lib.check(r)
    return dirty


def dirty2ms_mixed(uvw, freq, dirty, wgt, fov_deg, epsilon, sigma=2.0, sign=-1):
    """Precision-split dirty2ms on HOST arrays; returns complex64 visibilities [nrow]."""
    import numpy as np

    uvw = np.ascontiguousarray(uvw, dtype=np.float64)
    d = np.ascontiguousarray(dirty, dtype=np.complex64)
    w = None if wgt is None else np.ascontiguousarray(np.asarray(wgt).reshape(-1), dtype=np.float32)
    vis = np.zeros(uvw.shape[0], dtype=np.complex64)
    r = _lib.load().cg_dirty2ms_mixed(uvw.shape[0], d.shape[0], d.shape[1], fov_deg, freq,
                                      uvw.ctypes.data, vis.ctypes.data,
                                      None if w is None else w.ctypes.data, d.ctypes.data, epsilon,
                                      sigma, sign)
    _lib.check(r)
    return vis


def release_cache():
    """Free the device workspace cached by the host-pointer entry points."""
    _lib.check(_lib.load().cg_release_cache())


def set_host_kernel(kind="es", W=0, coef=None):
    """Gridding kernel of the host-pointer entry points (the reference-named
    functions and *_mixed): "es" (W = 0: from epsilon, the reference's choice)
    or "poly" with a [W, 8] Horner table, e.g. a learned kernel."""
    import numpy as np

    lib = _lib.load()
    if kind == "es":
        _lib.check(lib.cg_set_host_kernel(_lib.CG_KERNEL_ES, int(W or 0), None))
        return
    a = np.ascontiguousarray(np.asarray(coef, dtype=np.float64).reshape(int(W), 8))
    _lib.check(lib.cg_set_host_kernel(_lib.CG_KERNEL_POLY, int(W), a.ctypes.data))
