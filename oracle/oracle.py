"""ctypes front end of the CPU oracle (oracle/cg_oracle.c).

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use this module as the checker.  The product
library never imports it.

The oracle restates the reference's improved W-stacking ms2dirty/dirty2ms
(RapidsAtHKUST/cuGridder ``src/astro/ra_exec.cu:184-680``) and the FP64
direct DFT of the reference's tests (``python/curagridder/test_wst.py:15-32``)
on the CPU.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


class Params(ctypes.Structure):
    """Mirror of ``og_params`` (the reference's plan scalars)."""

    _fields_ = [
        ("nrow", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("N1", ctypes.c_int), ("N2", ctypes.c_int),
        ("fov", ctypes.c_double), ("freq", ctypes.c_double),
        ("eps", ctypes.c_double), ("sigma", ctypes.c_double),
        ("sign", ctypes.c_int),
        ("kw", ctypes.c_int),
        ("beta", ctypes.c_double), ("es_c", ctypes.c_double), ("es_halfwidth", ctypes.c_double),
        ("nf1", ctypes.c_int), ("nf2", ctypes.c_int), ("nf3", ctypes.c_int),
        ("pixelsize_x", ctypes.c_double), ("pixelsize_y", ctypes.c_double),
        ("i_center", ctypes.c_double), ("i_half_width", ctypes.c_double),
        ("o_center", ctypes.c_double), ("o_half_width", ctypes.c_double),
        ("gamma", ctypes.c_double), ("h", ctypes.c_double),
        ("hivesize", ctypes.c_int * 3), ("nhive", ctypes.c_int * 3),
        ("kern", ctypes.c_int), ("poly", ctypes.c_double * (16 * 8)),
    ]

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if not isinstance(v, (int, float)) else v
        return d


def build():
    """Compile oracle/_build/liboracle.so (plain gcc, no GPU needed)."""
    subprocess.check_call(["make", "-s", "-C", _HERE], stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "cg_oracle.c"))
        ):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        D = ctypes.POINTER(ctypes.c_double)
        I64 = ctypes.POINTER(ctypes.c_int64)
        I32 = ctypes.POINTER(ctypes.c_int)
        P = ctypes.POINTER(Params)
        L.og_setup.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                               ctypes.c_double, D, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                               ctypes.c_double]
        L.og_next235beven.argtypes = [ctypes.c_int, ctypes.c_int]
        L.og_grid_coords.argtypes = [P, D, D, D, D]
        L.og_bin_keys.argtypes = [P, D, I64]
        L.og_bin_mapping.argtypes = [P, D, I64, I32]
        L.og_gauss_legendre.argtypes = [ctypes.c_int, D, D]
        L.og_fseries_uv.argtypes = [P, ctypes.c_int, D]
        L.og_fseries_w.argtypes = [P, D, D]
        L.og_grid.argtypes = [P, D, D, D, D, D]
        L.og_degrid.argtypes = [P, D, D, D, D, D]
        L.og_fft2_planes.argtypes = [P, D, ctypes.c_int]
        for fn in (L.og_ms2dirty, L.og_dirty2ms):
            fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                           D, D, D, D, ctypes.c_double, ctypes.c_double, ctypes.c_int, P]
        for fn in (L.og_dft_ms2dirty, L.og_dft_dirty2ms):
            fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                           D, D, D, ctypes.c_int, ctypes.c_int, I64, D]
        L.og_num_threads.restype = ctypes.c_int
        L.og_set_kernel.argtypes = [ctypes.c_int, ctypes.c_int, D]
        L.og_learn_phi.argtypes = [D, ctypes.c_double, ctypes.c_int, ctypes.c_int, D, D]
        L.og_learn_phi_grad.argtypes = [D, ctypes.c_double, ctypes.c_int, ctypes.c_int, D, D, D]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _f64c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def setup(uvw, nx, ny, fov, freq, eps, sigma=2.0, sign=-1, eps_floor=1.1e-16):
    uvw = _f64c(uvw)
    p = Params()
    ier = lib().og_setup(ctypes.byref(p), uvw.shape[0], nx, ny, fov, freq, _d(uvw), eps, sigma,
                         sign, eps_floor)
    if ier > 1:
        raise ValueError("oracle setup error %d" % ier)
    return p


def next235beven(n, b=1):
    return lib().og_next235beven(n, b)


def grid_coords(p, uvw):
    uvw = _f64c(uvw)
    n = uvw.shape[0]
    X = np.zeros((3, n))
    lib().og_grid_coords(ctypes.byref(p), _d(uvw), _d(X[0]), _d(X[1]), _d(X[2]))
    return X


def bin_keys(p, uvw):
    uvw = _f64c(uvw)
    k = np.zeros(uvw.shape[0], dtype=np.int64)
    lib().og_bin_keys(ctypes.byref(p), _d(uvw),
                      k.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    return k


def bin_mapping(p, uvw):
    """(hive_start[nhive+1] int64, perm[nrow] int32) of the reference's bin_mapping."""
    uvw = _f64c(uvw)
    nh = p.nhive[0] * p.nhive[1] * p.nhive[2]
    hs = np.zeros(nh + 1, dtype=np.int64)
    perm = np.zeros(uvw.shape[0], dtype=np.int32)
    lib().og_bin_mapping(ctypes.byref(p), _d(uvw),
                         hs.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                         perm.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    return hs, perm


def gauss_legendre(n):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().og_gauss_legendre(n, _d(x), _d(w))
    return x, w


def fseries_uv(p, nf):
    out = np.zeros(nf // 2 + 1)
    lib().og_fseries_uv(ctypes.byref(p), nf, _d(out))
    return out


def fseries_w(p):
    nq = (p.N2 // 2 + 1) * (p.N1 // 2 + 1)
    out = np.zeros(nq)
    zp = np.zeros(nq)
    lib().og_fseries_w(ctypes.byref(p), _d(out), _d(zp))
    return out, zp


def grid(p, X, c, out=None):
    """Periodic ES spreading; returns fw [nf3, nf2, nf1] complex128 (written
    into `out` when given: a C-contiguous complex128 array of that shape)."""
    c = _c128(c)
    X = _f64c(X)
    if out is not None:
        assert out.dtype == np.complex128 and out.flags.c_contiguous
        assert out.shape == (p.nf3, p.nf2, p.nf1)
        fw = out
    else:
        fw = np.zeros((p.nf3, p.nf2, p.nf1), dtype=np.complex128)
    lib().og_grid(ctypes.byref(p), _d(X[0]), _d(X[1]), _d(X[2]), _d(c.view(np.float64)),
                  _d(fw.view(np.float64)))
    return fw


def degrid(p, X, fw):
    X = _f64c(X)
    fw = _c128(fw)
    c = np.zeros(X.shape[1], dtype=np.complex128)
    lib().og_degrid(ctypes.byref(p), _d(X[0]), _d(X[1]), _d(X[2]), _d(fw.view(np.float64)),
                    _d(c.view(np.float64)))
    return c


def fft2_planes(p, fw, sign):
    fw = _c128(fw).copy()
    lib().og_fft2_planes(ctypes.byref(p), _d(fw.view(np.float64)), sign)
    return fw


def ms2dirty(uvw, vis, wgt, nx, ny, fov, freq, eps, sigma=2.0, sign=-1):
    """Restated reference ms2dirty_2 / ms2dirty_1 (FP64); returns (dirty[nx,ny], params)."""
    uvw = _f64c(uvw)
    vis = _c128(vis)
    dirty = np.zeros((nx, ny), dtype=np.complex128)
    p = Params()
    w = _f64c(wgt) if wgt is not None else None
    ier = lib().og_ms2dirty(uvw.shape[0], nx, ny, fov, freq, _d(uvw), _d(vis.view(np.float64)),
                            _d(w) if w is not None else None, _d(dirty.view(np.float64)), eps,
                            sigma, sign, ctypes.byref(p))
    if ier > 1:
        raise ValueError("oracle ms2dirty error %d" % ier)
    return dirty, p


def dirty2ms(uvw, dirty, wgt, fov, freq, eps, sigma=2.0, sign=-1):
    """Restated reference dirty2ms_2 / dirty2ms_1 (FP64); returns (vis[nrow], params)."""
    uvw = _f64c(uvw)
    dirty = _c128(dirty)
    nx, ny = dirty.shape
    vis = np.zeros(uvw.shape[0], dtype=np.complex128)
    p = Params()
    w = _f64c(wgt) if wgt is not None else None
    ier = lib().og_dirty2ms(uvw.shape[0], nx, ny, fov, freq, _d(uvw), _d(vis.view(np.float64)),
                            _d(w) if w is not None else None, _d(dirty.view(np.float64)), eps,
                            sigma, sign, ctypes.byref(p))
    if ier > 1:
        raise ValueError("oracle dirty2ms error %d" % ier)
    return vis, p


def dft_ms2dirty(uvw, vis, wgt, nx, ny, fov, freq, sign=-1, pixels=None):
    """FP64 direct DFT image (all pixels, or the flat pixel indices given)."""
    uvw = _f64c(uvw)
    vis = _c128(vis)
    w = _f64c(wgt) if wgt is not None else None
    if pixels is None:
        out = np.zeros(nx * ny, dtype=np.complex128)
        npix, pp = -1, None
    else:
        pixels = np.ascontiguousarray(pixels, dtype=np.int64)
        out = np.zeros(pixels.size, dtype=np.complex128)
        npix, pp = pixels.size, pixels.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    lib().og_dft_ms2dirty(uvw.shape[0], nx, ny, fov, freq, _d(uvw), _d(vis.view(np.float64)),
                          _d(w) if w is not None else None, sign, npix, pp,
                          _d(out.view(np.float64)))
    return out.reshape(nx, ny) if pixels is None else out


def dft_dirty2ms(uvw, dirty, wgt, fov, freq, sign=-1, rows=None):
    """FP64 direct adjoint DFT visibilities (all rows, or the rows given)."""
    uvw = _f64c(uvw)
    dirty = _c128(dirty)
    nx, ny = dirty.shape
    w = _f64c(wgt) if wgt is not None else None
    if rows is None:
        out = np.zeros(uvw.shape[0], dtype=np.complex128)
        nv, rp = -1, None
    else:
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        out = np.zeros(rows.size, dtype=np.complex128)
        nv, rp = rows.size, rows.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    lib().og_dft_dirty2ms(uvw.shape[0], nx, ny, fov, freq, _d(uvw), _d(dirty.view(np.float64)),
                          _d(w) if w is not None else None, sign, nv, rp,
                          _d(out.view(np.float64)))
    return out


def num_threads():
    return lib().og_num_threads()


# ---------------------------------------------------------------- learned kernel
def set_kernel(kind="es", W=0, coef=None):
    """Kernel used by every following setup / ms2dirty / dirty2ms call:
    "es" (the reference's) or "poly" (piecewise Horner table [W, 8])."""
    if kind == "es":
        lib().og_set_kernel(0, 0, None)
        return
    a = np.ascontiguousarray(np.asarray(coef, dtype=np.float64).reshape(int(W), 8))
    lib().og_set_kernel(1, int(W), _d(a))


def learn_phi(theta, beta0, W, d):
    th = _f64c(theta)
    d = _f64c(d)
    out = np.zeros_like(d)
    lib().og_learn_phi(_d(th), float(beta0), int(W), d.size, _d(d), _d(out))
    return out


def learn_phi_grad(theta, beta0, W, d, dphi):
    th = _f64c(theta)
    d = _f64c(d)
    g = _f64c(dphi)
    out = np.zeros_like(th)
    lib().og_learn_phi_grad(_d(th), float(beta0), int(W), d.size, _d(d), _d(g), _d(out))
    return out
