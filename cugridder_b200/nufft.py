"""Generic type-1 / type-2 NUFFT in 1-3 dimensions on device arrays (the
reference's cunufft front end, src/fourier/cuft.cu:327-545).

    p = NufftPlan(type=1, nmodes=(N1, N2), iflag=+1, eps=1e-6, precision="fp64")
    p.setpts(x, y)            # torch CUDA float64 arrays, radians
    p.execute(c, fk)          # type 1: c [M] -> fk [N2, N1]; type 2: fk -> c
"""
import ctypes

import numpy as np

from . import _lib


class NufftPlan:
    def __init__(self, type, nmodes, iflag=1, eps=1e-6, sigma=2.0, precision="fp64", stream=None):
        self._lib = _lib.load()
        self.dim = len(nmodes)
        self.nmodes = tuple(int(n) for n in nmodes)
        prec = _lib.CG_PREC_FP32 if precision in ("fp32", "f32") else _lib.CG_PREC_FP64
        nm = (ctypes.c_int64 * 3)(*(list(self.nmodes) + [1] * (3 - self.dim)))
        h = ctypes.c_void_p()
        if stream is None:
            try:
                import torch

                stream = torch.cuda.current_stream().cuda_stream if torch.cuda.is_available() else None
            except Exception:
                stream = None
        _lib.check(self._lib.cg_nufft_create(ctypes.byref(h), int(type), self.dim,
                                             ctypes.addressof(nm), int(iflag), float(eps),
                                             float(sigma), prec, stream))
        self._h = h
        self._pts = None

    def setpts(self, x, y=None, z=None):
        self._pts = (x, y, z)  # the coordinate arrays are read during setpts only
        _lib.check(self._lib.cg_nufft_setpts(self._h, int(x.shape[0]), _lib.ptr(x), _lib.ptr(y),
                                             _lib.ptr(z)))

    def execute(self, c, fk):
        return _lib.check(self._lib.cg_nufft_execute(self._h, _lib.ptr(c), _lib.ptr(fk)))

    def info(self):
        kw = ctypes.c_int()
        nf = (ctypes.c_int64 * 3)()
        _lib.check(self._lib.cg_nufft_get_info(self._h, ctypes.byref(kw), ctypes.addressof(nf)))
        return {"kw": kw.value, "nf": list(nf)}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cg_nufft_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
