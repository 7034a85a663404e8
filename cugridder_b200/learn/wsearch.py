"""Smallest kernel width W that meets a target accuracy, for ES and for the
learned kernels, measured through the full FP32 W-stacking pipeline.

    python -m cugridder_b200.learn.wsearch [--nrow 10000000] [--out kernels/wsearch_2048_10M.json]

Workload: 2048 x 2048 image, fov 3 deg, 10M visibilities at 1.5e8 Hz,
u, v ~ N(0, 4000 m) clipped to +-16 km, w ~ U(-1 km, 1 km), complex64, sigma 2
(the evaluation set of the kernel study).  For W = 4..10 it runs ms2dirty and
dirty2ms with ES at width W (the reference's beta for that W) and with each
trained kernel, and measures the relative L2 error against the FP64 direct
sums computed on the device (cg_explicit_*) on random pixel and row subsets.
A kernel meets epsilon at W when both directions' errors are <= epsilon.
"""
import argparse
import json
import os
import time

import numpy as np

from .. import Plan, _lib, synth
from .model import KERNEL_DIR, available_widths, load_kernel


def _stream(torch):
    return torch.cuda.current_stream().cuda_stream


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


class Reference:
    """FP64 direct sums of one dataset on random pixel / row subsets (device DFT)."""

    def __init__(self, torch, d, img, npix, nrows, seed=0):
        lib = _lib.load()
        nx, ny = d["nx"], d["ny"]
        rng = np.random.Generator(np.random.PCG64(seed))
        self.pix = np.sort(rng.choice(nx * ny, npix, replace=False)).astype(np.int64)
        self.rows = np.sort(rng.choice(d["uvw"].shape[0], nrows, replace=False)).astype(np.int64)
        dev = torch.device("cuda")
        uvw = torch.from_numpy(d["uvw"]).to(dev)
        vis = torch.from_numpy(d["vis"].astype(np.complex128)).to(dev)
        wgt = torch.from_numpy(d["wgt"].astype(np.float64)).to(dev)
        dimg = torch.from_numpy(img.astype(np.complex128)).to(dev)
        pix = torch.from_numpy(self.pix).to(dev)
        rows = torch.from_numpy(self.rows).to(dev)
        out = torch.empty(npix, dtype=torch.complex128, device=dev)
        vout = torch.empty(nrows, dtype=torch.complex128, device=dev)
        M = d["uvw"].shape[0]
        t0 = time.time()
        _lib.check(lib.cg_explicit_ms2dirty(M, nx, ny, d["fov"], d["freq"], uvw.data_ptr(),
                                            vis.data_ptr(), wgt.data_ptr(), -1, npix, pix.data_ptr(),
                                            out.data_ptr(), _stream(torch)))
        _lib.check(lib.cg_explicit_dirty2ms(M, nx, ny, d["fov"], d["freq"], uvw.data_ptr(),
                                            dimg.data_ptr(), wgt.data_ptr(), -1, nrows,
                                            rows.data_ptr(), vout.data_ptr(), _stream(torch)))
        torch.cuda.synchronize()
        self.seconds = time.time() - t0
        self.dirty = out.cpu().numpy()
        self.vis = vout.cpu().numpy()


def run_kernel(torch, d, img, kernel, W, coef=None, precision="fp32", eps=1e-5, reps=2):
    """ms2dirty + dirty2ms with one kernel; returns (dirty, vis, ms per direction, info)."""
    dev = torch.device("cuda")
    cdt = torch.complex64 if precision == "fp32" else torch.complex128
    rdt = torch.float32 if precision == "fp32" else torch.float64
    plan = Plan(d["nx"], d["ny"], d["fov"], eps, precision=precision)
    plan.set_kernel(kernel, W, coef)
    uvw = torch.from_numpy(d["uvw"]).to(dev)
    vis = torch.from_numpy(d["vis"]).to(device=dev, dtype=cdt)
    wgt = torch.from_numpy(d["wgt"]).to(device=dev, dtype=rdt)
    dimg = torch.from_numpy(img).to(device=dev, dtype=cdt)
    dirty = torch.empty((d["nx"], d["ny"]), dtype=cdt, device=dev)
    vout = torch.empty(d["uvw"].shape[0], dtype=cdt, device=dev)
    times = []
    for _ in range(reps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        plan.ms2dirty(uvw, d["freq"], vis, wgt, dirty)
        e[1].record()
        plan.dirty2ms(uvw, d["freq"], dimg, wgt, vout)
        e[2].record()
        torch.cuda.synchronize()
        times.append((e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])))
    info = plan.info()
    plan.close()
    return dirty.cpu().numpy(), vout.cpu().numpy(), times[-1], info


def search(torch, nrow=10_000_000, widths=range(4, 11), eps_list=(1e-4, 1e-5, 1e-6), npix=1024,
           nrows=1024, kernel_dir=None, log=print):
    d = synth.make("wstack_2048_10M", seed=0, nrow=nrow)
    img = synth.random_image(d["nx"], d["ny"], seed=1, dtype=np.complex64)
    ref = Reference(torch, d, img, npix, nrows, seed=2)
    log("direct sums: %.1f s" % ref.seconds)
    learned = set(available_widths(kernel_dir))
    results = []
    for W in widths:
        kinds = [("es", None)]
        if W in learned:
            kinds.append(("learned", load_kernel(W, kernel_dir).horner))
        for name, coef in kinds:
            dirty, vis, ms, info = run_kernel(torch, d, img, "es" if name == "es" else "poly", W, coef)
            r = {"kernel": name, "W": W, "nw": info["nw"],
                 "err_ms2dirty": rel_l2(dirty.reshape(-1)[ref.pix], ref.dirty),
                 "err_dirty2ms": rel_l2(vis[ref.rows], ref.vis),
                 "ms_ms2dirty": round(ms[0], 3), "ms_dirty2ms": round(ms[1], 3)}
            results.append(r)
            log(json.dumps(r))
    best = {}
    for eps in eps_list:
        best["%g" % eps] = {}
        for name in ("es", "learned"):
            ok = [r["W"] for r in results if r["kernel"] == name and
                  max(r["err_ms2dirty"], r["err_dirty2ms"]) <= eps]
            best["%g" % eps][name] = min(ok) if ok else None
    return {
        "workload": {"name": "wstack_2048_10M", "nx": d["nx"], "ny": d["ny"], "fov_deg": d["fov"],
                     "nrow": nrow, "freq_hz": d["freq"], "precision": "fp32 (fp64 uvw)",
                     "reference": "FP64 direct sums on the device on %d pixels / %d rows" % (npix, nrows)},
        "criterion": "relative L2 error of ms2dirty and of dirty2ms both <= epsilon",
        "results": results, "smallest_W": best,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nrow", type=int, default=10_000_000)
    ap.add_argument("--out", default=os.path.join(KERNEL_DIR, "wsearch_2048_10M.json"))
    ap.add_argument("--kernels", default=None, help="directory of learned_W*.json (default: the package's)")
    a = ap.parse_args()
    import torch

    res = search(torch, nrow=a.nrow, kernel_dir=a.kernels)
    with open(a.out, "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps(res["smallest_W"]))


if __name__ == "__main__":
    main()
