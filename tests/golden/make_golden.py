"""Record golden outputs of the REFERENCE's own CUDA library.

Runs oracle/_ref/libcurafft_ref.so -- the reference's sources compiled for
sm_100a by oracle/ref.mk -- through its own C entry points (ms2dirty_2,
dirty2ms_2, ms2dirtyf_2, dirty2msf_2; reference src/astro/cugridder.cu:541-571)
on seeded inputs, and writes the outputs with the input checksums to an .npz.
Needs a CUDA GPU and the reference build:

    python tests/golden/make_golden.py --out tests/golden/ref_golden.npz

The tests regenerate the inputs from the seeds (cugridder_b200.synth) and
check the checksums.
"""
import argparse
import ctypes
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from cugridder_b200 import synth  # noqa: E402

P = ctypes.c_void_p


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        if a is not None:
            h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def cases():
    """(name, precision, inputs) of every golden case."""
    out = []
    c1 = synth.make("ms2dirty_256_fp64", seed=0)
    img = synth.random_image(256, 256, seed=1)
    out.append(("c1_fp64", "fp64", dict(uvw=c1["uvw"], vis=c1["vis"], wgt=c1["wgt"], dirty_in=img,
                                          nx=256, ny=256, fov=2.0, freq=1.0e8, eps=1e-5, sign=-1,
                                          keep_vis=8192)))
    out.append(("c1_fp32", "fp32", dict(uvw=c1["uvw"].astype(np.float32),
                                          vis=c1["vis"].astype(np.complex64),
                                          wgt=c1["wgt"].astype(np.float32),
                                          dirty_in=img.astype(np.complex64), nx=256, ny=256,
                                          fov=2.0, freq=1.0e8, eps=1e-5, sign=-1, keep_vis=8192)))
    for single in (False, True):
        t = synth.test_wst_case(100, 32, 128, fov=10, seed=42, single=single)
        dt = np.complex64 if single else np.complex128
        rt = np.float32 if single else np.float64
        d_in = np.zeros((32, 128), dtype=dt)
        d_in.real = t["dirty"]
        out.append(("wst_100_32x128_" + ("fp32" if single else "fp64"), "fp32" if single else "fp64",
                    dict(uvw=t["uvw"].astype(rt), vis=t["ms"].astype(dt), wgt=t["wgt"].astype(rt),
                         dirty_in=d_in, nx=32, ny=128, fov=10.0, freq=1e9, eps=5e-5, sign=-1,
                         keep_vis=100)))
    t = synth.test_wst_case(1000, 64, 64, fov=5, seed=7, use_wgt=False)
    d_in = np.zeros((64, 64), dtype=np.complex128)
    d_in.real = t["dirty"]
    out.append(("ws_1000_64x64_sign+1_fp64", "fp64",
                dict(uvw=t["uvw"], vis=t["ms"], wgt=None, dirty_in=d_in, nx=64, ny=64, fov=5.0,
                     freq=1e9, eps=1e-7, sign=1, keep_vis=1000)))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--lib", default=os.path.join(ROOT, "oracle", "_ref", "libcurafft_ref.so"))
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden", "ref_golden.npz"))
    a = ap.parse_args()
    lib = ctypes.CDLL(a.lib)
    D, F, I = ctypes.c_double, ctypes.c_float, ctypes.c_int
    fns = {}
    for name, real in (("ms2dirty_2", D), ("dirty2ms_2", D), ("ms2dirty_1", D), ("dirty2ms_1", D),
                       ("ms2dirtyf_2", F), ("dirty2msf_2", F), ("ms2dirtyf_1", F),
                       ("dirty2msf_1", F)):
        f = getattr(lib, name)
        wg = name.endswith("_2")
        f.argtypes = [I, I, I, real, real, P, P] + ([P] if wg else []) + [P, real, real, I]
        f.restype = I
        fns[name] = f
    rec = {}
    for name, prec, c in cases():
        sfx = "f" if prec == "fp32" else ""
        wg = c["wgt"] is not None
        uvw = np.ascontiguousarray(c["uvw"])
        vis = np.ascontiguousarray(c["vis"])
        nrow = uvw.shape[0]
        dirty = np.zeros((c["nx"], c["ny"]), dtype=vis.dtype)
        args = [nrow, c["nx"], c["ny"], c["fov"], c["freq"], uvw.ctypes.data, vis.ctypes.data]
        if wg:
            wgt = np.ascontiguousarray(c["wgt"])
            args.append(wgt.ctypes.data)
        args += [dirty.ctypes.data, c["eps"], 2.0, c["sign"]]
        r1 = fns["ms2dirty%s_%d" % (sfx, 2 if wg else 1)](*args)
        vout = np.zeros(nrow, dtype=vis.dtype)
        d_in = np.ascontiguousarray(c["dirty_in"])
        args = [nrow, c["nx"], c["ny"], c["fov"], c["freq"], uvw.ctypes.data, vout.ctypes.data]
        if wg:
            args.append(wgt.ctypes.data)
        args += [d_in.ctypes.data, c["eps"], 2.0, c["sign"]]
        r2 = fns["dirty2ms%s_%d" % (sfx, 2 if wg else 1)](*args)
        rec[name + "/dirty"] = dirty
        rec[name + "/vis"] = vout[: c["keep_vis"]]
        rec[name + "/status"] = np.array([r1, r2])
        rec[name + "/sha_inputs"] = np.array(sha(uvw, vis, c["wgt"], d_in))
        print(name, "status", r1, r2, "dirty norm", np.linalg.norm(dirty), "vis norm",
              np.linalg.norm(vout), flush=True)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    np.savez_compressed(a.out, **rec)
    print("wrote", a.out)


if __name__ == "__main__":
    main()
