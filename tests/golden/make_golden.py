"""Record golden outputs of the REFERENCE's own CUDA library.

Runs oracle/_ref/libcurafft_ref.so -- the reference's sources compiled for
sm_100a by oracle/ref.mk -- through its own C entry points (ms2dirty_2,
dirty2ms_2, ms2dirtyf_2, dirty2msf_2; reference src/astro/cugridder.cu:541-571)
on seeded inputs, and writes the outputs with the input checksums to an .npz.
Needs a CUDA GPU and the reference build:

    python tests/golden/make_golden.py --out tests/golden/ref_golden.npz
    python tests/golden/make_golden.py --bins-out tests/golden/ref_bins.npz
    python tests/golden/make_golden.py --large-out tests/golden/ref_large.npz
    python tests/golden/make_golden.py --add-dft tests/golden/ref_large.npz   (CPU)

--bins-out runs the reference's binning stage through oracle/ref_bins.cu
(oracle/_ref/libref_bins.so) and keeps its hive offsets and per-cell row
counts; --large-out keeps the full-size outputs on 4096-pixel / 4096-row
subsets.

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


def canon_cells(keys, counts):
    """sha256 of a per-cell row count list in canonical form: the nonzero
    cells' keys ascending as little-endian uint64, then their counts as int32."""
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(keys, dtype="<u8").tobytes())
    h.update(np.ascontiguousarray(counts, dtype="<i4").tobytes())
    return h.hexdigest()


def bin_cases():
    """(name, inputs) of the binning records: c1, a grid whose axes are not
    multiples of 8 cells with rows over the whole band and past it, and the
    first 1M rows of the 4096^2 workload at its full geometry."""
    c1 = synth.make("ms2dirty_256_fp64", seed=0)
    wr = synth.wrap_case(50_000, 122, 250, 3.0, seed=31)
    c2 = synth.make("wstack_4096_20M", seed=0, nrow=1_000_000)
    return [("c1", dict(uvw=c1["uvw"], nx=256, ny=256, fov=2.0, freq=1.0e8, eps=1e-5, full=True)),
            ("wrap_122x250", dict(uvw=wr["uvw"], nx=122, ny=250, fov=3.0, freq=1.0e9, eps=1e-6,
                                  full=True)),
            ("c2_1M", dict(uvw=c2["uvw"], nx=4096, ny=4096, fov=5.0, freq=1.5e8, eps=1e-5,
                           full=False))]


def record_bins(out):
    """The reference's binning (oracle/_ref/libref_bins.so: its gridder_setting
    + cura_prestage -> bin_mapping, FP64 build) on bin_cases()."""
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_bins.so"))
    fn = lib.refbins_ms2dirty
    I, D, L = ctypes.c_int, ctypes.c_double, ctypes.c_longlong
    fn.argtypes = [I, I, I, D, D, P, D, D, I, P, P, P, L, P, P, L, P, P]
    fn.restype = I
    rec = {}
    for name, c in bin_cases():
        uvw = np.ascontiguousarray(c["uvw"], dtype=np.float64)
        nrow = uvw.shape[0]
        nf = np.zeros(3, np.int32)
        nh = np.zeros(3, np.int32)
        method = np.zeros(1, np.int32)
        ncells = np.zeros(1, np.int64)
        hcap = 64 << 20
        hive = np.zeros(hcap, np.int32)
        keys = np.zeros(nrow, np.uint64)
        cnts = np.zeros(nrow, np.int32)
        r = fn(nrow, c["nx"], c["ny"], c["fov"], c["freq"], uvw.ctypes.data, c["eps"], 2.0, -1,
               nf.ctypes.data, nh.ctypes.data, hive.ctypes.data, hcap, keys.ctypes.data,
               cnts.ctypes.data, nrow, ncells.ctypes.data, method.ctypes.data)
        n = int(ncells[0])
        nhv = int(nh[0]) * int(nh[1]) * int(nh[2])
        hive = hive[: nhv + 1]
        keys, cnts = keys[:n], cnts[:n]
        print("bins", name, "status", r, "nf", nf, "nhive", nh, "method", int(method[0]),
              "cells", n, "rows", int(cnts.sum()), flush=True)
        rec[name + "/status"] = np.array(r)
        rec[name + "/nf"] = nf
        rec[name + "/nhive"] = nh
        rec[name + "/method"] = method
        rec[name + "/ncells"] = np.array(n)
        rec[name + "/cells_sha"] = np.array(canon_cells(keys, cnts))
        rec[name + "/hive_sha"] = np.array(hashlib.sha256(hive.astype("<i4").tobytes()).hexdigest())
        rec[name + "/sha_uvw"] = np.array(sha(uvw))
        if c["full"]:
            rec[name + "/hive_count"] = hive
    np.savez_compressed(out, **rec)
    print("wrote", out)


def large_cases():
    """(name, config, nrow, eps list) of the full-size records."""
    return [("c2", "wstack_4096_20M", 20_000_000, [("fp32", 1e-5), ("fp64", 1e-5), ("fp64", 1e-9)]),
            ("c4", "wstack_2048_10M", 10_000_000, [("fp32", 1e-5), ("fp64", 1e-5), ("fp64", 1e-4)])]


def record_large(fns, out, nsub=4096):
    """The reference's own ms2dirty / dirty2ms (host API, its FP32 build with
    FP32 coordinates and its FP64 build) at full size on the 4096^2 / 20M and
    2048^2 / 10M workloads (seed 0, the image of seed 1000 as bench.py uses),
    kept on a seeded random subset of nsub pixels and nsub rows."""
    import time

    rec = {}
    for name, cfg, nrow, runs in large_cases():
        d = synth.make(cfg, seed=0, nrow=nrow)
        img = synth.random_image(d["nx"], d["ny"], seed=1000, dtype=np.complex64)
        rng = np.random.Generator(np.random.PCG64(4242))
        pix = np.sort(rng.choice(d["nx"] * d["ny"], nsub, replace=False)).astype(np.int64)
        rows = np.sort(rng.choice(nrow, nsub, replace=False)).astype(np.int64)
        rec[name + "/pixels"] = pix
        rec[name + "/rows"] = rows
        rec[name + "/sha_inputs"] = np.array(sha(d["uvw"], d["vis"], d["wgt"], img))
        for prec, eps in runs:
            single = prec == "fp32"
            rt, ct = (np.float32, np.complex64) if single else (np.float64, np.complex128)
            uvw = np.ascontiguousarray(d["uvw"], dtype=rt)
            vis = np.ascontiguousarray(d["vis"], dtype=ct)
            wgt = np.ascontiguousarray(d["wgt"], dtype=rt)
            dimg = np.ascontiguousarray(img, dtype=ct)
            dirty = np.zeros((d["nx"], d["ny"]), dtype=ct)
            vout = np.zeros(nrow, dtype=ct)
            sfx = "f" if single else ""
            t0 = time.perf_counter()
            r1 = fns["ms2dirty%s_2" % sfx](nrow, d["nx"], d["ny"], d["fov"], d["freq"],
                                           uvw.ctypes.data, vis.ctypes.data, wgt.ctypes.data,
                                           dirty.ctypes.data, eps, 2.0, -1)
            t1 = time.perf_counter()
            r2 = fns["dirty2ms%s_2" % sfx](nrow, d["nx"], d["ny"], d["fov"], d["freq"],
                                           uvw.ctypes.data, vout.ctypes.data, wgt.ctypes.data,
                                           dimg.ctypes.data, eps, 2.0, -1)
            t2 = time.perf_counter()
            key = "%s/%s_%g" % (name, prec, eps)
            rec[key + "/status"] = np.array([r1, r2])
            rec[key + "/dirty"] = dirty.reshape(-1)[pix].astype(np.complex128)
            rec[key + "/vis"] = vout[rows].astype(np.complex128)
            rec[key + "/seconds"] = np.array([t1 - t0, t2 - t1])
            print(key, "status", r1, r2, "seconds %.2f %.2f" % (t1 - t0, t2 - t1), flush=True)
            del uvw, vis, wgt, dimg, dirty, vout
    np.savez_compressed(out, **rec)
    print("wrote", out)


def add_dft(path):
    """Add the oracle's FP64 direct sums (CPU, oracle/cg_oracle.c) on the
    recorded pixel / row subsets of each full-size case to the .npz at path,
    and print the reference's own errors against them.  CPU only."""
    from oracle import oracle as O

    from cugridder_b200.synth import rel_l2

    rec = dict(np.load(path))
    for name, cfg, nrow, runs in large_cases():
        d = synth.make(cfg, seed=0, nrow=nrow)
        img = synth.random_image(d["nx"], d["ny"], seed=1000, dtype=np.complex64)
        assert sha(d["uvw"], d["vis"], d["wgt"], img) == str(rec[name + "/sha_inputs"])
        pix, rows = rec[name + "/pixels"], rec[name + "/rows"]
        rec[name + "/dft_dirty"] = O.dft_ms2dirty(d["uvw"], d["vis"], d["wgt"], d["nx"], d["ny"],
                                                 d["fov"], d["freq"], pixels=pix)
        rec[name + "/dft_vis"] = O.dft_dirty2ms(d["uvw"], img, d["wgt"], d["fov"], d["freq"],
                                               rows=rows)
        for prec, eps in runs:
            key = "%s/%s_%g" % (name, prec, eps)
            print(key, "reference vs DFT: dirty %.3e vis %.3e" % (
                rel_l2(rec[key + "/dirty"], rec[name + "/dft_dirty"]),
                rel_l2(rec[key + "/vis"], rec[name + "/dft_vis"])), flush=True)
    np.savez_compressed(path, **rec)
    print("wrote", path)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--lib", default=os.path.join(ROOT, "oracle", "_ref", "libcurafft_ref.so"))
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden", "ref_golden.npz"))
    ap.add_argument("--bins-out", default=None,
                    help="record the reference's binning (libref_bins.so) to this .npz and exit")
    ap.add_argument("--large-out", default=None,
                    help="record the full-size 4096^2 / 2048^2 subsets to this .npz and exit")
    ap.add_argument("--add-dft", default=None,
                    help="add the oracle's CPU direct sums on the subsets to this --large-out "
                         ".npz (no GPU needed) and exit")
    a = ap.parse_args()
    if a.add_dft:
        add_dft(a.add_dft)
        return
    if a.bins_out:
        record_bins(a.bins_out)
        return
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
    if a.large_out:
        record_large(fns, a.large_out)
        return
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
