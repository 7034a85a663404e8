"""Reusable plan over DEVICE buffers (torch CUDA tensors or raw addresses).

Replaces the reference's gridder_setting / gridder_execution / gridder_destroy
trio (src/astro/cugridder.cu:90-257), which rebuilds plan and workspace on
every call, with a plan whose HBM workspace and cuFFT plan persist.

    plan = Plan(nxdirty, nydirty, fov_deg, epsilon, precision="fp32")
    plan.ms2dirty(uvw, freq, vis, wgt, dirty)   # all CUDA tensors
    plan.dirty2ms(uvw, freq, dirty, wgt, vis)

Layouts: uvw float64 [nrow, 3]; fp64 plans take complex128 vis/dirty and
float64 wgt, fp32 plans complex64 vis/dirty and float32 wgt.  Calls are
ordered on the plan's stream (by default torch's current stream).
"""
import ctypes

import numpy as np

from . import _lib


def _default_stream():
    try:
        import torch

        if torch.cuda.is_available():
            return torch.cuda.current_stream().cuda_stream
    except Exception:
        pass
    return None


class Plan:
    def __init__(self, nxdirty, nydirty, fov_deg, epsilon, sigma=2.0, sign=-1, precision="fp32",
                 stream=None):
        self._lib = _lib.load()
        self.precision = _lib.CG_PREC_FP32 if precision in ("fp32", "f32", 1) else _lib.CG_PREC_FP64
        self.nxdirty, self.nydirty = int(nxdirty), int(nydirty)
        h = ctypes.c_void_p()
        st = stream if stream is not None else _default_stream()
        r = self._lib.cg_plan_create(ctypes.byref(h), self.nxdirty, self.nydirty, float(fov_deg),
                                     float(epsilon), float(sigma), int(sign), self.precision, st)
        _lib.check(r)
        self.status = r
        self._h = h

    def set_stream(self, stream):
        _lib.check(self._lib.cg_plan_set_stream(self._h, stream))

    def ms2dirty(self, uvw, freq, vis, wgt, dirty, nrow=None):
        n = int(nrow if nrow is not None else uvw.shape[0])
        r = self._lib.cg_plan_ms2dirty(self._h, n, float(freq), _lib.ptr(uvw), _lib.ptr(vis),
                                       _lib.ptr(wgt), _lib.ptr(dirty))
        return _lib.check(r)

    def dirty2ms(self, uvw, freq, dirty, wgt, vis, nrow=None):
        n = int(nrow if nrow is not None else uvw.shape[0])
        r = self._lib.cg_plan_dirty2ms(self._h, n, float(freq), _lib.ptr(uvw), _lib.ptr(dirty),
                                       _lib.ptr(wgt), _lib.ptr(vis))
        return _lib.check(r)

    def ms2dirty_chan(self, uvw, freqs, vis, wgt, dirty):
        """Multi-channel ms2dirty: vis / wgt [nrow, nchan] on the device, freqs
        a host sequence of nchan frequencies; every channel is summed into dirty."""
        f = np.ascontiguousarray(np.asarray(freqs, dtype=np.float64).reshape(-1))
        r = self._lib.cg_plan_ms2dirty_chan(self._h, int(uvw.shape[0]), f.size, f.ctypes.data,
                                            _lib.ptr(uvw), _lib.ptr(vis), _lib.ptr(wgt),
                                            _lib.ptr(dirty))
        return _lib.check(r)

    def dirty2ms_chan(self, uvw, freqs, dirty, wgt, vis):
        """Multi-channel dirty2ms into vis [nrow, nchan] on the device."""
        f = np.ascontiguousarray(np.asarray(freqs, dtype=np.float64).reshape(-1))
        r = self._lib.cg_plan_dirty2ms_chan(self._h, int(uvw.shape[0]), f.size, f.ctypes.data,
                                            _lib.ptr(uvw), _lib.ptr(dirty), _lib.ptr(wgt),
                                            _lib.ptr(vis))
        return _lib.check(r)

    def info(self):
        inf = _lib.PlanInfo()
        _lib.check(self._lib.cg_plan_get_info(self._h, ctypes.byref(inf)))
        return inf.as_dict()

    def set_method(self, method):
        """1 = tiled SIMT (default), 2 = tensor-core gridding where supported, 0 = direct."""
        _lib.check(self._lib.cg_plan_set_method(self._h, int(method)))

    def set_kernel(self, kind="es", W=None, coef=None):
        """Gridding kernel: "es" (W from epsilon, or forced when W is given) or
        "poly" with width W and a [W, 8] array of piecewise Horner coefficients
        (a learned kernel, see cugridder_b200.learn)."""
        if kind == "es":
            _lib.check(self._lib.cg_plan_set_kernel(self._h, _lib.CG_KERNEL_ES, int(W or 0), None))
            return
        a = np.ascontiguousarray(np.asarray(coef, dtype=np.float64).reshape(int(W), 8))
        _lib.check(self._lib.cg_plan_set_kernel(self._h, _lib.CG_KERNEL_POLY, int(W), a.ctypes.data))

    def set_autotune(self, on=True):
        """Time candidate tilings on the first call per direction and keep the fastest."""
        _lib.check(self._lib.cg_plan_set_autotune(self._h, 1 if on else 0))

    def tiling(self):
        """(gridding x, y, planes, warps), (degridding x, y, planes, threads), tuned ms."""
        t = (ctypes.c_int * 8)()
        ms = (ctypes.c_float * 2)()
        _lib.check(self._lib.cg_plan_get_tiling(self._h, ctypes.addressof(t), ctypes.addressof(ms)))
        return tuple(t[:4]), tuple(t[4:]), (ms[0], ms[1])

    def set_fixed_uvw(self, on=True):
        """Reuse geometry and binning while uvw (same array), nrow and freq stay fixed."""
        _lib.check(self._lib.cg_plan_set_fixed_uvw(self._h, 1 if on else 0))

    def set_grid_budget(self, nbytes):
        """Memory-limited mode: keep at most nbytes of w planes resident (0: no limit)."""
        _lib.check(self._lib.cg_plan_set_grid_budget(self._h, int(nbytes)))

    def set_stop_stage(self, stage):
        _lib.check(self._lib.cg_plan_set_stop_stage(self._h, int(stage)))

    def check_status(self):
        """Wait for the plan's stream; raise GridderError if a bounded TMA
        staging wait of the degridding ran out since the last check."""
        return _lib.check(self._lib.cg_plan_status(self._h))

    def copy_buffer(self, which):
        """Copy an internal buffer (CG_BUF_*) of the last call to a numpy array."""
        need = ctypes.c_size_t()
        _lib.check(self._lib.cg_plan_copy_buffer(self._h, which, None, 0, ctypes.byref(need)))
        cplx = np.complex128 if self.precision == _lib.CG_PREC_FP64 else np.complex64
        dt = {
            _lib.CG_BUF_HIVE_START: np.int32, _lib.CG_BUF_PERM: np.int32,
            _lib.CG_BUF_SORTED_KEYS: np.int64, _lib.CG_BUF_GRID: cplx,
            _lib.CG_BUF_FSERIES_1: np.float64, _lib.CG_BUF_FSERIES_2: np.float64,
            _lib.CG_BUF_FSERIES_W: np.float64,
        }[which]
        out = np.empty(need.value // np.dtype(dt).itemsize, dtype=dt)
        _lib.check(self._lib.cg_plan_copy_buffer(self._h, which, out.ctypes.data, out.nbytes,
                                                 ctypes.byref(need)))
        if which == _lib.CG_BUF_GRID:
            inf = self.info()
            out = out.reshape(inf["nw"], inf["nf2"], inf["nf1"])
        return out

    MS2DIRTY_STAGES = ["w_range", "quarter_tables", "binning", "sorted_stream", "gridding", "fft",
                       "wdft_deconv"]
    DIRTY2MS_STAGES = ["w_range", "quarter_tables", "binning", "plane_fill", "fft",
                       "sorted_stream", "degridding"]

    def set_timing(self, on=True):
        """Enable per-stage CUDA-event timers (resets the totals)."""
        _lib.check(self._lib.cg_plan_set_timing(self._h, 1 if on else 0))

    def timing(self):
        """{"ms2dirty": {stage: total ms}, "dirty2ms": {...}, "calls": (n0, n1)}"""
        out = {}
        calls = []
        for d, names in ((0, self.MS2DIRTY_STAGES), (1, self.DIRTY2MS_STAGES)):
            buf = (ctypes.c_double * 8)()
            n = ctypes.c_int()
            nc = ctypes.c_longlong()
            _lib.check(self._lib.cg_plan_get_timing(self._h, d, buf, 8, ctypes.byref(n),
                                                    ctypes.byref(nc)))
            out["ms2dirty" if d == 0 else "dirty2ms"] = {names[i]: buf[i] for i in range(n.value)}
            calls.append(nc.value)
        out["calls"] = tuple(calls)
        return out

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cg_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
