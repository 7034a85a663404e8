"""Batched solves on device tensors: many datasets (own image size, fov,
rows, channels) per call, all spread / interpolated by one persistent
launch whose tiling is autotuned on the first call; the second call per
direction is captured into a CUDA graph and later calls replay it.

    b = Batch([dict(uvw=uvw, freqs=[f0, f1], vis=vis, wgt=wgt, dirty=dirty, fov=2.0), ...],
              epsilon=1e-4, precision="fp32")
    b.ms2dirty()          # images of every dataset into its `dirty`
    b.dirty2ms()          # visibilities of every dataset into its `vis`

The tensors must stay alive and uvw unchanged for the life of the batch.
"""
import ctypes

import numpy as np

from . import _lib


class _Dataset(ctypes.Structure):
    _fields_ = [("nrow", ctypes.c_int64), ("nchan", ctypes.c_int),
                ("freqs", ctypes.POINTER(ctypes.c_double)), ("nxdirty", ctypes.c_int),
                ("nydirty", ctypes.c_int), ("fov", ctypes.c_double), ("d_uvw", ctypes.c_void_p),
                ("d_vis", ctypes.c_void_p), ("d_wgt", ctypes.c_void_p),
                ("d_dirty", ctypes.c_void_p)]


class Batch:
    def __init__(self, datasets, epsilon, sigma=2.0, sign=-1, precision="fp32", stream=None):
        self._lib = _lib.load()
        self._keep = datasets
        arr = (_Dataset * len(datasets))()
        self._freqs = []
        for i, d in enumerate(datasets):
            f = np.ascontiguousarray(np.asarray(d["freqs"], dtype=np.float64).reshape(-1))
            self._freqs.append(f)
            arr[i].nrow = int(d["uvw"].shape[0])
            arr[i].nchan = int(f.size)
            arr[i].freqs = f.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            arr[i].nxdirty, arr[i].nydirty = int(d["dirty"].shape[0]), int(d["dirty"].shape[1])
            arr[i].fov = float(d["fov"])
            arr[i].d_uvw = _lib.ptr(d["uvw"])
            arr[i].d_vis = _lib.ptr(d["vis"])
            arr[i].d_wgt = _lib.ptr(d.get("wgt"))
            arr[i].d_dirty = _lib.ptr(d["dirty"])
        if stream is None:
            import torch

            stream = torch.cuda.current_stream().cuda_stream
        prec = _lib.CG_PREC_FP32 if precision in ("fp32", "f32") else _lib.CG_PREC_FP64
        h = ctypes.c_void_p()
        _lib.check(self._lib.cg_batch_create(ctypes.byref(h), len(datasets), ctypes.addressof(arr),
                                             float(epsilon), float(sigma), int(sign), prec, stream))
        self._h = h

    def ms2dirty(self):
        _lib.check(self._lib.cg_batch_ms2dirty(self._h))

    def dirty2ms(self):
        _lib.check(self._lib.cg_batch_dirty2ms(self._h))

    def set_kernel(self, kind="es", W=None, coef=None):
        """Gridding kernel of every dataset (as Plan.set_kernel); before the first call."""
        if kind == "es":
            _lib.check(self._lib.cg_batch_set_kernel(self._h, _lib.CG_KERNEL_ES, int(W or 0), None))
            return
        a = np.ascontiguousarray(np.asarray(coef, dtype=np.float64).reshape(int(W), 8))
        _lib.check(self._lib.cg_batch_set_kernel(self._h, _lib.CG_KERNEL_POLY, int(W), a.ctypes.data))

    def tiling(self):
        """Autotuned tiling: (gridding x, y, planes, warps), (degridding x,
        y, planes, threads) and the winning launch times in ms (0 = default
        / not tuned yet)."""
        t = (ctypes.c_int * 8)()
        ms = (ctypes.c_float * 2)()
        _lib.check(self._lib.cg_batch_get_tiling(self._h, ctypes.addressof(t), ctypes.addressof(ms)))
        return tuple(t[:4]), tuple(t[4:]), (ms[0], ms[1])

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
