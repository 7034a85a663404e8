"""Time the REFERENCE's own CUDA build on the GPU, through its own C entry
points, on the benchmark workload (and a smaller one).

Runs oracle/_ref/libcurafft_ref.so (the reference's sources compiled for
sm_100a by oracle/ref.mk) with ms2dirty_2 + dirty2ms_2 (FP64) and
ms2dirtyf_2 + dirty2msf_2 (its -DSINGLE build, FP32 coordinates too) on the
same seeded data as bench.py, host pointers in and out as the reference's API
takes them, and prints one JSON line per case with Mvis/s =
nrow / (t_ms2dirty + t_dirty2ms).  Needs a CUDA GPU:

    python tests/golden/time_reference_build.py --out tests/golden/reference_gpu_b200.json
"""
import argparse
import ctypes
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from cugridder_b200 import synth  # noqa: E402

P = ctypes.c_void_p


def bind(lib):
    D, F, I = ctypes.c_double, ctypes.c_float, ctypes.c_int
    out = {}
    for name, real in (("ms2dirty_2", D), ("dirty2ms_2", D), ("ms2dirtyf_2", F), ("dirty2msf_2", F)):
        f = getattr(lib, name)
        f.argtypes = [I, I, I, real, real, P, P, P, P, real, real, I]
        f.restype = I
        out[name] = f
    return out


def run_case(fns, cfg, nrow, precision, eps, reps):
    d = synth.make(cfg, seed=0, nrow=nrow)
    img = synth.random_image(d["nx"], d["ny"], seed=1000)
    single = precision == "fp32"
    rt, ct = (np.float32, np.complex64) if single else (np.float64, np.complex128)
    uvw = np.ascontiguousarray(d["uvw"], dtype=rt)
    vis = np.ascontiguousarray(d["vis"], dtype=ct)
    wgt = np.ascontiguousarray(d["wgt"], dtype=rt)
    dimg = np.ascontiguousarray(img, dtype=ct)
    dirty = np.zeros((d["nx"], d["ny"]), dtype=ct)
    vout = np.zeros(nrow, dtype=ct)
    f1, f2 = (fns["ms2dirtyf_2"], fns["dirty2msf_2"]) if single else (fns["ms2dirty_2"], fns["dirty2ms_2"])
    times = []
    for r in range(reps + 1):
        t0 = time.perf_counter()
        s1 = f1(nrow, d["nx"], d["ny"], d["fov"], d["freq"], uvw.ctypes.data, vis.ctypes.data,
                wgt.ctypes.data, dirty.ctypes.data, eps, 2.0, -1)
        t1 = time.perf_counter()
        s2 = f2(nrow, d["nx"], d["ny"], d["fov"], d["freq"], uvw.ctypes.data, vout.ctypes.data,
                wgt.ctypes.data, dimg.ctypes.data, eps, 2.0, -1)
        t2 = time.perf_counter()
        if r > 0:  # the first call pays the CUDA context and module loading
            times.append((t1 - t0, t2 - t1))
    t_m, t_d = (float(np.median([t[i] for t in times])) for i in (0, 1))
    return {"impl": "reference CUDA build (oracle/_ref, sm_100a)", "workload": cfg, "nrow": nrow,
            "nx": d["nx"], "ny": d["ny"], "precision": precision, "eps": eps,
            "status": [int(s1), int(s2)], "ms2dirty_s": round(t_m, 4), "dirty2ms_s": round(t_d, 4),
            "mvis_per_s": round(nrow / (t_m + t_d) / 1e6, 3), "reps": reps,
            "timing": "host wall clock around each synchronous call (its API: host buffers)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--lib", default=os.path.join(ROOT, "oracle", "_ref", "libcurafft_ref.so"))
    ap.add_argument("--out", default=None)
    ap.add_argument("--reps", type=int, default=2)
    a = ap.parse_args()
    fns = bind(ctypes.CDLL(a.lib))
    res = []
    for cfg, nrow in (("wstack_2048_10M", 2_000_000), ("wstack_4096_20M", 20_000_000)):
        for prec in ("fp32", "fp64"):
            r = run_case(fns, cfg, nrow, prec, 1e-5, a.reps)
            print(json.dumps(r), flush=True)
            res.append(r)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
