"""Loader of libcugridder.so (the sm_100a CUDA library) with ctypes signatures.

The library is built in-tree (``python -m cugridder_b200.build``).  If it is
missing, one build is attempted; if that fails the import fails loudly --
there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libcugridder.so")

c_int, c_double, c_float, c_void_p, c_int64, c_size_t = (
    ctypes.c_int, ctypes.c_double, ctypes.c_float, ctypes.c_void_p, ctypes.c_int64,
    ctypes.c_size_t)

CG_PREC_FP64 = 0
CG_PREC_FP32 = 1
CG_BUF_HIVE_START = 1
CG_BUF_PERM = 2
CG_BUF_SORTED_KEYS = 3
CG_BUF_GRID = 4
CG_BUF_FSERIES_1 = 5
CG_BUF_FSERIES_2 = 6
CG_BUF_FSERIES_W = 7
CG_KERNEL_ES = 0
CG_KERNEL_POLY = 1

STATUS = {
    0: "ok", 1: "epsilon clipped to the precision floor", 2: "invalid argument",
    3: "CUDA error", 4: "cuFFT error", 5: "device memory exhausted",
    6: "problem too large", 7: "no CUDA device",
}


class GridderError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__("cugridder error %d (%s)%s" % (code, STATUS.get(code, "?"),
                                                         (": " + msg) if msg else ""))
        self.code = code


class PlanInfo(ctypes.Structure):
    _fields_ = [
        ("kw", c_int), ("beta", c_double), ("nf1", c_int), ("nf2", c_int), ("nw", c_int),
        ("i_center", c_double), ("i_half_width", c_double), ("o_center", c_double),
        ("o_half_width", c_double), ("gamma", c_double), ("h", c_double),
        ("pixelsize_x", c_double), ("pixelsize_y", c_double), ("nhive", c_int * 3),
        ("nrow", c_int64), ("workspace_bytes", c_size_t),
    ]

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if name == "nhive" else v
        return d


# exported symbols, with (restype, argtypes)
_PTR = c_void_p
SIGNATURES = {
    "ms2dirty_2": (c_int, [c_int, c_int, c_int, c_double, c_double, _PTR, _PTR, _PTR, _PTR, c_double, c_double, c_int]),
    "ms2dirty_1": (c_int, [c_int, c_int, c_int, c_double, c_double, _PTR, _PTR, _PTR, c_double, c_double, c_int]),
    "dirty2ms_1": (c_int, [c_int, c_int, c_int, c_double, c_double, _PTR, _PTR, _PTR, c_double, c_double, c_int]),
    "dirty2ms_2": (c_int, [c_int, c_int, c_int, c_double, c_double, _PTR, _PTR, _PTR, _PTR, c_double, c_double, c_int]),
    "ms2dirtyf_2": (c_int, [c_int, c_int, c_int, c_float, c_float, _PTR, _PTR, _PTR, _PTR, c_float, c_float, c_int]),
    "ms2dirtyf_1": (c_int, [c_int, c_int, c_int, c_float, c_float, _PTR, _PTR, _PTR, c_float, c_float, c_int]),
    "dirty2msf_1": (c_int, [c_int, c_int, c_int, c_float, c_float, _PTR, _PTR, _PTR, c_float, c_float, c_int]),
    "dirty2msf_2": (c_int, [c_int, c_int, c_int, c_float, c_float, _PTR, _PTR, _PTR, _PTR, c_float, c_float, c_int]),
    "cg_ms2dirty_mixed": (c_int, [c_int64, c_int, c_int, c_double, c_double, _PTR, _PTR, _PTR, _PTR, c_double, c_double, c_int]),
    "cg_dirty2ms_mixed": (c_int, [c_int64, c_int, c_int, c_double, c_double, _PTR, _PTR, _PTR, _PTR, c_double, c_double, c_int]),
    "cg_plan_create": (c_int, [ctypes.POINTER(c_void_p), c_int, c_int, c_double, c_double, c_double, c_int, c_int, c_void_p]),
    "cg_plan_set_stream": (c_int, [c_void_p, c_void_p]),
    "cg_plan_ms2dirty": (c_int, [c_void_p, c_int64, c_double, _PTR, _PTR, _PTR, _PTR]),
    "cg_plan_dirty2ms": (c_int, [c_void_p, c_int64, c_double, _PTR, _PTR, _PTR, _PTR]),
    "cg_plan_get_info": (c_int, [c_void_p, ctypes.POINTER(PlanInfo)]),
    "cg_plan_ms2dirty_chan": (c_int, [c_void_p, c_int64, c_int, _PTR, _PTR, _PTR, _PTR, _PTR]),
    "cg_plan_dirty2ms_chan": (c_int, [c_void_p, c_int64, c_int, _PTR, _PTR, _PTR, _PTR, _PTR]),
    "cg_plan_destroy": (c_int, [c_void_p]),
    "cg_plan_copy_buffer": (c_int, [c_void_p, c_int, c_void_p, c_size_t, ctypes.POINTER(c_size_t)]),
    "cg_plan_set_stop_stage": (c_int, [c_void_p, c_int]),
    "cg_plan_status": (c_int, [c_void_p]),
    "cg_plan_set_grid_budget": (c_int, [c_void_p, c_size_t]),
    "cg_plan_set_fixed_uvw": (c_int, [c_void_p, c_int]),
    "cg_plan_set_method": (c_int, [c_void_p, c_int]),
    "cg_plan_set_timing": (c_int, [c_void_p, c_int]),
    "cg_plan_get_timing": (c_int, [c_void_p, c_int, ctypes.POINTER(c_double), c_int,
                                   ctypes.POINTER(c_int), ctypes.POINTER(ctypes.c_longlong)]),
    "cg_bin_static": (c_int, [c_int64, c_int, c_int, c_double, c_double, _PTR, c_double, c_double,
                              c_int, c_int, _PTR, _PTR, c_int64, ctypes.POINTER(c_int64), c_void_p]),
    "cg_bin_static_max_rows": (c_int64, []),
    "cg_plan_set_kernel": (c_int, [c_void_p, c_int, c_int, _PTR]),
    "cg_set_host_kernel": (c_int, [c_int, c_int, _PTR]),
    "cg_learn_theta_size": (c_int, []),
    "cg_learn_phi_forward": (c_int, [_PTR, c_float, c_int, c_int64, _PTR, _PTR, c_void_p]),
    "cg_learn_phi_backward": (c_int, [_PTR, c_float, c_int, c_int64, _PTR, _PTR, _PTR, c_void_p]),
    "cg_learn_spread2d": (c_int, [c_int, c_int, c_int, c_int, _PTR, _PTR, _PTR, _PTR, _PTR, _PTR,
                                  c_void_p]),
    "cg_learn_spread2d_adjoint": (c_int, [c_int, c_int, c_int, c_int, _PTR, _PTR, _PTR, _PTR, _PTR,
                                          _PTR, _PTR, _PTR, c_void_p]),
    "cg_learn_dft2": (c_int, [c_int, c_int, c_int, _PTR, _PTR, _PTR, c_int, _PTR, _PTR, _PTR,
                              c_void_p]),
    "cg_explicit_ms2dirty": (c_int, [c_int64, c_int, c_int, c_double, c_double, _PTR, _PTR, _PTR,
                                     c_int, c_int64, _PTR, _PTR, c_void_p]),
    "cg_explicit_dirty2ms": (c_int, [c_int64, c_int, c_int, c_double, c_double, _PTR, _PTR, _PTR,
                                     c_int, c_int64, _PTR, _PTR, c_void_p]),
    "cg_nufft_create": (c_int, [ctypes.POINTER(c_void_p), c_int, c_int, _PTR, c_int, c_double,
                                c_double, c_int, c_void_p]),
    "cg_nufft_setpts": (c_int, [c_void_p, c_int64, _PTR, _PTR, _PTR]),
    "cg_nufft_execute": (c_int, [c_void_p, _PTR, _PTR]),
    "cg_nufft_get_info": (c_int, [c_void_p, ctypes.POINTER(c_int), _PTR]),
    "cg_nufft_destroy": (c_int, [c_void_p]),
    "cg_batch_create": (c_int, [ctypes.POINTER(c_void_p), c_int, _PTR, c_double, c_double, c_int,
                                c_int, c_void_p]),
    "cg_batch_ms2dirty": (c_int, [c_void_p]),
    "cg_batch_dirty2ms": (c_int, [c_void_p]),
    "cg_batch_destroy": (c_int, [c_void_p]),
    "cg_batch_get_tiling": (c_int, [c_void_p, c_void_p, c_void_p]),
    "cg_batch_set_kernel": (c_int, [c_void_p, c_int, c_int, c_void_p]),
    "cg_plan_set_autotune": (c_int, [c_void_p, c_int]),
    "cg_plan_get_tiling": (c_int, [c_void_p, c_void_p, c_void_p]),
    "cg_release_cache": (c_int, []),
    "cg_last_error": (ctypes.c_char_p, []),
    "cg_kernel_launches": (ctypes.c_longlong, []),
    "cg_version": (c_int, []),
}

_lib = None


def load():
    """Return the loaded CDLL; build it once if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build
        try:
            _build.build()
        except Exception as e:  # no silent fallback
            raise ImportError("libcugridder.so is missing and could not be built: %s" % e)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(code, allow_warning=True):
    if code == 0 or (code == 1 and allow_warning):
        return code
    msg = load().cg_last_error()
    raise GridderError(code, msg.decode() if msg else "")


def ptr(a):
    """Raw address of a numpy array, a torch tensor, an int or None."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    raise TypeError("cannot take the address of %r" % type(a))
