#!/usr/bin/env python
"""Benchmark: Mvis/s of ms2dirty + dirty2ms (improved W-stacking) on B200.

One step = ms2dirty of the workload's visibilities followed by dirty2ms of an
image onto the same rows (Mvis/s = nrow / (t_ms2dirty + t_dirty2ms) / 1e6).
Default workload: 4096x4096 image, fov 5 deg, 20M rows at 1.5e8 Hz,
u,v ~ N(0, 6000 m) clipped to +-20 km, w ~ U(-2 km, 2 km), complex64
visibilities, float32 weights, FP64 uvw, epsilon 1e-5 -- the precision-split
FP32 form; the plain FP64 form of the same workload is measured beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 runs under torchrun, one process per GPU, each on its own synthetic
dataset (weak scaling, no collective on the data path); the time is the max
over ranks.  --impl reference times the reference algorithm on the host cores
(the CPU restatement in oracle/, all threads), on a bounded sample of the same
workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "wstack_4096_20M"
METRIC = "Mvis/s ms2dirty+dirty2ms at eps 1e-5, learned-FP32 vs plain ES-FP64, 1 B200"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default=WORKLOAD)
    ap.add_argument("--nrow", type=int, default=None, help="override the number of rows")
    ap.add_argument("--fov", type=float, default=None,
                    help="override the field of view in degrees (fewer w planes: small profiling cases)")
    ap.add_argument("--eps", type=float, default=1e-5)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default tilings (no autotuning on the first call)")
    ap.add_argument("--batch", action="store_true",
                    help="the batched workload: 32 uneven datasets (synth.batch_specs), eps 1e-4")
    ap.add_argument("--kernel", default="auto", choices=["auto", "es", "learned"],
                    help="auto: the learned kernel at the smallest width that met epsilon in the "
                         "committed width search, else ES")
    ap.add_argument("--accuracy-samples", type=int, default=256,
                    help="pixels / rows checked against the FP64 direct sums (0: skip)")
    ap.add_argument("--eps-fp64-leg", type=float, default=1e-9,
                    help="epsilon of the workload's FP64 leg, timed beside the main line (0: skip)")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched workload's forms in the main line")
    ap.add_argument("--ref-reps", type=int, default=3,
                    help="timed calls of the reference's CUDA build (--impl reference)")
    ap.add_argument("--_ref-cuda-worker", dest="ref_cuda_worker", action="store_true",
                    help=argparse.SUPPRESS)
    return ap.parse_args()


def select_kernel(args):
    """Gridding kernel of the FP32 form: the learned kernel at the smallest W
    that met epsilon in cugridder_b200/kernels/wsearch_2048_10M.json, else ES."""
    from cugridder_b200.learn import available_widths, load_kernel
    from cugridder_b200.learn.model import KERNEL_DIR

    es = {"kind": "es", "W": 0, "coef": None, "label": "ES (W from epsilon)"}
    if args.kernel == "es":
        return es
    p = os.path.join(KERNEL_DIR, "wsearch_2048_10M.json")
    W = None
    if os.path.exists(p):
        with open(p) as f:
            best = json.load(f).get("smallest_W", {})
        W = (best.get("%g" % args.eps) or {}).get("learned")
    if W is None or W not in available_widths():
        if args.kernel == "learned":
            raise SystemExit("no learned kernel meets eps %g" % args.eps)
        return es
    k = load_kernel(W)
    return {"kind": "poly", "W": W, "coef": k.horner,
            "label": "learned MLP kernel, W=%d, piecewise degree-7 Horner" % W}


# --------------------------------------------------------------------------- ranks
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if (torch.cuda.is_available() and dist.get_backend() == "nccl") else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if (torch.cuda.is_available() and dist.get_backend() == "nccl") else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(s[1]) for s in self.samples if num(s[1]) is not None]
        mx = [num(s[2]) for s in self.samples if num(s[2]) is not None]
        power = [num(s[3]) for s in self.samples if num(s[3]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i] == "Active"})
        loaded = [x for x, p in zip(sm, power) if p is not None and p > 250] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "power_w_max": max(power) if power else None, "samples": len(self.samples)}


# --------------------------------------------------------------------------- peaks
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel, workload):
    """Per-launch DRAM traffic recorded from an ncu capture (profiles/*.json)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(workload, {}).get(kernel)


# --------------------------------------------------------------------------- workload
def workload_config(args, world):
    """The workload's defining parameters: the same dict in both arms'
    lines (implementation details are reported under "impl_detail")."""
    from cugridder_b200 import synth

    cfg = synth.CONFIGS[args.config]
    return {"workload": args.config, "nx": cfg["nx"], "ny": cfg["ny"],
            "fov_deg": args.fov or cfg["fov"], "nrow_per_gpu": args.nrow or cfg["nrow"],
            "freq_hz": cfg["freq"], "eps": args.eps, "sigma": 2.0, "sign": -1,
            "uv_sigma_m": cfg["uv_sigma"], "uv_clip_m": cfg["uv_clip"], "w_max_m": cfg["w_max"],
            "parallelism": "independent datasets per GPU" if world > 1 else "single GPU",
            "l2": "inputs larger than L2 (uvw 480 MB, grid 7.5 GB)"}


def make_data(cfg_name, seed, nrow, torch, fov=None):
    from cugridder_b200 import synth

    over = {"fov": fov} if fov else {}
    d = synth.make(cfg_name, seed=seed, nrow=nrow, **over)
    img = synth.random_image(d["nx"], d["ny"], seed=seed + 1000, dtype=np.complex64)
    return d, img


def fft_cells(d, info):
    """Cells the band-pruned transform reads plus writes per w plane: the row
    transforms over the grid rows that hold data (read and written whole,
    batch rounded up to 64 rows as the plan does) and the column transforms
    over the image columns, reading the band's rows and writing the image's
    rows (ms2dirty; dirty2ms moves the same cells the other way)."""
    nf1, nf2, W = info["nf1"], info["nf2"], info["kw"]
    u = d["uvw"][:, 0] * (d["freq"] / 299792458.0)
    pixx = np.deg2rad(d["fov"]) / d["nx"]
    span = (float(u.max()) - float(u.min())) * pixx * nf2 + W + 1
    nb = min(nf2, int(np.ceil(span / 64.0)) * 64)
    return 2 * nb * nf1 + nb * d["ny"] + d["nx"] * d["ny"]


def algorithmic_bytes(stage, d, info, prec):
    """Minimum HBM bytes of one launch of each stage (reads of its inputs plus
    writes of its outputs, each once)."""
    M = d["uvw"].shape[0]
    s_c = 8 if prec == "fp32" else 16
    rec = 32 if prec == "fp32" else 48
    G = info["nf1"] * info["nf2"] * info["nw"]
    npix = d["nx"] * d["ny"]
    nq = (d["nx"] // 2 + 1) * (d["ny"] // 2 + 1)
    # FP32 power-of-two grids: the forward column kernel does not load the rows
    # outside the image in the image's columns, and the plane fill skips them
    fill_cells = G
    if prec == "fp32" and info["nf2"] in (1024, 2048, 4096, 8192):
        fill_cells = (info["nf1"] * info["nf2"] - (info["nf2"] - d["nx"]) * d["ny"]) * info["nw"]
    return {
        "gridding": M * rec + G * s_c,
        "degridding": G * s_c + M * rec + M * 4 + M * s_c,
        "plane_fill": fill_cells * s_c + npix * s_c + nq * 16,
        "wdft_deconv": info["nw"] * npix * s_c + npix * s_c + nq * 16,
        "fft": fft_cells(d, info) * info["nw"] * s_c,
        "sorted_stream": M * (4 + 24 + s_c + s_c // 2) + M * rec,
        "binning": M * 24 + 4 * 3 * M * 8,
    }.get(stage)


def run_b200(args, rank, world, local):
    import torch

    from cugridder_b200 import Plan, _lib, dirty2ms_mixed, ms2dirty_mixed, synth  # noqa: F401

    torch.cuda.set_device(local)
    if not args.no_autotune:  # the host entry points' cached plans too (e2e)
        os.environ["CG_AUTOTUNE"] = "1"
    cfg = synth.CONFIGS[args.config]
    d, img = make_data(args.config, rank, args.nrow, torch, args.fov)
    M = d["uvw"].shape[0]
    nx, ny, fov, freq = d["nx"], d["ny"], d["fov"], d["freq"]
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()

    uvw = torch.from_numpy(d["uvw"]).to(dev)
    res = {}
    lib = _lib.load()
    clocks = ClockSampler(local)

    rng = np.random.Generator(np.random.PCG64(77))
    nsamp = max(0, min(args.accuracy_samples, M, nx * ny))
    pix = np.sort(rng.choice(nx * ny, nsamp, replace=False)).astype(np.int64)
    rows = np.sort(rng.choice(M, nsamp, replace=False)).astype(np.int64)
    kern = select_kernel(args)

    def timed_run(prec, steps, warmup, sample_clocks=False, timing=False, kernel=None):
        cdt = torch.complex64 if prec == "fp32" else torch.complex128
        rdt = torch.float32 if prec == "fp32" else torch.float64
        vis = torch.from_numpy(d["vis"]).to(device=dev, dtype=cdt)
        wgt = torch.from_numpy(d["wgt"]).to(device=dev, dtype=rdt)
        dimg = torch.from_numpy(img).to(device=dev, dtype=cdt)
        dirty = torch.empty((nx, ny), dtype=cdt, device=dev)
        vout = torch.empty(M, dtype=cdt, device=dev)
        plan = Plan(nx, ny, fov, args.eps, precision=prec, stream=stream.cuda_stream)
        if kernel is not None and kernel["kind"] == "poly":
            plan.set_kernel("poly", kernel["W"], kernel["coef"])
        plan.set_autotune(not args.no_autotune)  # tuned in the first warm-up step

        def step():
            plan.ms2dirty(uvw, freq, vis, wgt, dirty)
            plan.dirty2ms(uvw, freq, dimg, wgt, vout)

        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        if timing:
            plan.set_timing(True)
        if sample_clocks:
            clocks.start()
            time.sleep(0.3)
        barrier(world)
        torch.cuda.synchronize()
        l0 = lib.cg_kernel_launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        launches = lib.cg_kernel_launches() - l0
        if sample_clocks:
            clocks.stop()
        ms = e0.elapsed_time(e1)
        # adjointness of the last step's pair: <dirty2ms(img), vis> = <img, ms2dirty(vis)>
        # (inner products in FP64, so that their own rounding does not enter)
        f64 = torch.complex128
        ip1 = complex(torch.vdot(vout.reshape(-1).to(f64), vis.reshape(-1).to(f64)).item())
        ip2 = complex(torch.vdot(dimg.reshape(-1).to(f64), dirty.reshape(-1).to(f64)).item())
        adjoint = abs(ip1 - ip2) / max(abs(ip1), abs(ip2), 1e-300)
        gt, dt, tms = plan.tiling()
        out = {"ms": ms, "launches": launches, "info": plan.info(), "adjointness": adjoint,
               "tiling": {"grid_warp_tile": list(gt), "degrid_tile": list(dt),
                          "tuned_launch_ms": [round(x, 3) for x in tms]}}
        if timing:
            out["timing"] = plan.timing()
        if nsamp:
            out["dirty_sub"] = dirty.reshape(-1).cpu().numpy()[pix].astype(np.complex128)
            out["vis_sub"] = vout.cpu().numpy()[rows].astype(np.complex128)
        plan.close()
        del vis, wgt, dimg, dirty, vout
        torch.cuda.empty_cache()
        return out

    main = timed_run("fp32", args.steps, args.warmup, sample_clocks=True, timing=True, kernel=kern)
    res["kernel"] = {"label": kern["label"], "W": main["info"]["kw"]}
    t_max = max_over_ranks(main["ms"], world)
    total_rows = sum_over_ranks(M, world)
    res["value"] = total_rows * args.steps / (t_max / 1e3) / 1e6
    res["ms_per_step"] = t_max / args.steps
    res["gpu_launches"] = int(main["launches"])
    res["info"] = main["info"]
    res["tiling"] = main["tiling"]
    res["adjointness"] = {"value_form": main["adjointness"]}

    # per-stage timing and roofline of the dominant kernel of this library
    tm = main["timing"]
    ncalls = max(tm["calls"][0], 1)
    stages = {}
    peak, peak_kind = measured_peaks()
    for direction in ("ms2dirty", "dirty2ms"):
        for name, total in tm[direction].items():
            per = total / ncalls
            b = algorithmic_bytes(name, d, main["info"], "fp32")
            stages[direction + "." + name] = {
                "ms": round(per, 4),
                "algorithmic_GB": None if b is None else round(b / 1e9, 4),
                "GBps": None if (b is None or per <= 0) else round(b / 1e9 / (per / 1e3), 1),
            }
    own = {k: v for k, v in stages.items() if not k.endswith(".fft") and not k.endswith("w_range")}
    dom = max(own, key=lambda k: own[k]["ms"])
    dom_name = dom.split(".")[1]
    ach = stages[dom]["GBps"]
    res["roofline"] = {
        "kernel": dom, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
        "frac": None if ach is None else round(ach / peak, 4),
        "traffic": ncu_traffic(dom_name, args.config), "peak_source": peak_kind,
    }
    res["stages"] = stages
    res["clocks"] = clocks.summary()

    if not args.no_fp64:
        fp = timed_run("fp64", max(2, args.steps // 3), args.warmup)
        res["adjointness"]["fp64_plain"] = fp["adjointness"]
        t64 = max_over_ranks(fp["ms"], world)
        v64 = total_rows * max(2, args.steps // 3) / (t64 / 1e3) / 1e6
        res["fp64_plain"] = {"value": round(v64, 2), "ms_per_step": round(t64 / max(2, args.steps // 3), 3),
                             "eps": args.eps, "kw": fp["info"]["kw"], "nw": fp["info"]["nw"]}
        res["fp32_over_fp64"] = round(res["value"] / v64, 3)
        if args.eps_fp64_leg > 0:
            # the workload's FP64 leg at its own epsilon (1e-9: W = 10)
            n9 = max(2, args.steps // 5)
            eps_main, args.eps = args.eps, args.eps_fp64_leg
            try:
                f9 = timed_run("fp64", n9, max(1, args.warmup - 1))
            finally:
                args.eps = eps_main
            t9 = max_over_ranks(f9["ms"], world)
            res["fp64_eps_leg"] = {"eps": args.eps_fp64_leg, "value": round(total_rows * n9 / (t9 / 1e3) / 1e6, 2),
                                   "ms_per_step": round(t9 / n9, 3), "kw": f9["info"]["kw"],
                                   "nw": f9["info"]["nw"], "adjointness": f9["adjointness"],
                                   "steps": n9}
            if nsamp:
                res["fp64_eps_leg"]["accuracy"] = accuracy(d, img, pix, rows, f9, None)["value_form"]

    if nsamp:
        res["accuracy"] = accuracy(d, img, pix, rows, main, fp if not args.no_fp64 else None)

    if not args.no_e2e:
        res["e2e"] = run_e2e(args, d, img, world, kern)

    if not args.no_batched and world == 1:
        # the batched workload: learned FP32 against plain ES FP64, both batched
        del uvw
        torch.cuda.empty_cache()
        eps_main, args.eps = args.eps, 1e-4
        try:
            bk = select_kernel(args)
            forms, meta, _ = batched_forms(args, bk, max(3, args.steps // 2), args.warmup,
                                           sequential=False)
        finally:
            args.eps = eps_main
        res["batched"] = {"config": meta, "learned_fp32": forms["learned_fp32"]["value"],
                          "es_fp32": forms["es_fp32"]["value"], "es_fp64": forms["es_fp64"]["value"],
                          "learned_fp32_over_es_fp64": round(forms["learned_fp32"]["value"] /
                                                             forms["es_fp64"]["value"], 3),
                          "forms": forms}
    return res


def accuracy(d, img, pix, rows, main, fp64):
    """Relative L2 error of each timed form against the FP64 direct sums
    (on-device explicit gridder) on random pixel / row subsets."""
    import torch

    from cugridder_b200 import _lib

    lib = _lib.load()
    dev = torch.device("cuda")
    M, nx, ny = d["uvw"].shape[0], d["nx"], d["ny"]
    st = torch.cuda.current_stream().cuda_stream
    uvw = torch.from_numpy(d["uvw"]).to(dev)
    vis = torch.from_numpy(d["vis"].astype(np.complex128)).to(dev)
    wgt = torch.from_numpy(d["wgt"].astype(np.float64)).to(dev)
    dimg = torch.from_numpy(img.astype(np.complex128)).to(dev)
    tp, tr = torch.from_numpy(pix).to(dev), torch.from_numpy(rows).to(dev)
    rd = torch.empty(pix.size, dtype=torch.complex128, device=dev)
    rv = torch.empty(rows.size, dtype=torch.complex128, device=dev)
    _lib.check(lib.cg_explicit_ms2dirty(M, nx, ny, d["fov"], d["freq"], uvw.data_ptr(), vis.data_ptr(),
                                        wgt.data_ptr(), -1, pix.size, tp.data_ptr(), rd.data_ptr(), st))
    _lib.check(lib.cg_explicit_dirty2ms(M, nx, ny, d["fov"], d["freq"], uvw.data_ptr(), dimg.data_ptr(),
                                        wgt.data_ptr(), -1, rows.size, tr.data_ptr(), rv.data_ptr(), st))
    torch.cuda.synchronize()
    ref_d, ref_v = rd.cpu().numpy(), rv.cpu().numpy()

    def err(r):
        return {"ms2dirty_rel_l2": float(np.linalg.norm(r["dirty_sub"] - ref_d) / np.linalg.norm(ref_d)),
                "dirty2ms_rel_l2": float(np.linalg.norm(r["vis_sub"] - ref_v) / np.linalg.norm(ref_v))}

    out = {"reference": "FP64 direct sums on the device (cg_explicit_*) on %d pixels / %d rows"
                        % (pix.size, rows.size), "value_form": err(main)}
    if fp64 is not None:
        out["fp64_plain"] = err(fp64)
    return out


def run_e2e(args, d, img, world, kern):
    """Same metric through the public host API (cg_ms2dirty_mixed /
    cg_dirty2ms_mixed, with the same gridding kernel selected by
    cg_set_host_kernel) from pinned host buffers: every step copies its inputs
    host->device and its outputs device->host."""
    import torch

    from cugridder_b200 import _lib, set_host_kernel

    lib = _lib.load()
    if kern["kind"] == "poly":
        set_host_kernel("poly", kern["W"], kern["coef"])
    M = d["uvw"].shape[0]
    nx, ny = d["nx"], d["ny"]

    def pinned(a):
        t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
        t.numpy()[...] = a
        return t.numpy()

    uvw = pinned(d["uvw"])
    vis = pinned(d["vis"].astype(np.complex64))
    wgt = pinned(d["wgt"].astype(np.float32))
    dimg = pinned(img.astype(np.complex64))
    dirty = pinned(np.zeros((nx, ny), np.complex64))
    vout = pinned(np.zeros(M, np.complex64))

    def step():
        r1 = lib.cg_ms2dirty_mixed(M, nx, ny, d["fov"], d["freq"], uvw.ctypes.data, vis.ctypes.data,
                                   wgt.ctypes.data, dirty.ctypes.data, args.eps, 2.0, -1)
        r2 = lib.cg_dirty2ms_mixed(M, nx, ny, d["fov"], d["freq"], uvw.ctypes.data, vout.ctypes.data,
                                   wgt.ctypes.data, dimg.ctypes.data, args.eps, 2.0, -1)
        _lib.check(r1)
        _lib.check(r2)

    step()
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(torch.cuda.default_stream())
    for _ in range(args.e2e_steps):
        step()
    e1.record(torch.cuda.default_stream())
    torch.cuda.synchronize()
    barrier(world)
    t = max_over_ranks(e0.elapsed_time(e1), world)
    total_rows = sum_over_ranks(M, world)
    lib.cg_release_cache()
    set_host_kernel("es")
    h2d = 2 * uvw.nbytes + vis.nbytes + 2 * wgt.nbytes + dimg.nbytes
    d2h = dirty.nbytes + vout.nbytes
    return {"value": round(total_rows * args.e2e_steps / (t / 1e3) / 1e6, 2), "unit": "Mvis/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "ms_per_step": round(t / args.e2e_steps, 3), "api": "cg_ms2dirty_mixed+cg_dirty2ms_mixed"}


# --------------------------------------------------------------------------- CPU (oracle port)
class CpuReference:
    """Mvis/s of the reference algorithm restated on the host cores (the
    oracle's C/OpenMP port, all threads) for the full workload, EXTRAPOLATED
    from measured parts:
      - gridding and degridding of a sample of rows on the workload's
        full-size grid (same nf, nw, W, so cache behaviour is the real one),
        per row, times the workload's rows, plus one zeroing of the grid;
      - one full-size 2-D FFT plane, times nw, per direction;
      - the per-pixel w stage and corrections of a 256^2 run, times the
        workload's pixels, per direction.
    The fixed-cost parts are measured once; each sample() times new rows."""

    def __init__(self, cfg_name):
        from cugridder_b200 import synth
        from oracle import oracle as O

        self.O = O
        self.cfg_name = cfg_name
        full = self.full = synth.CONFIGS[cfg_name]
        # geometry of the full workload (its w range is +-w_max)
        self.p = O.setup(np.array([[0, 0, -full["w_max"]], [0, 0, full["w_max"]]], float),
                         full["nx"], full["ny"], full["fov"], full["freq"], 1e-5)
        p = self.p
        self.fw = np.empty((p.nf3, p.nf2, p.nf1), dtype=np.complex128)
        p0 = type(p).from_buffer_copy(p)
        p0.nrow = 0
        none = np.zeros((3, 0))
        O.grid(p0, none, np.zeros(0, np.complex128), out=self.fw)  # first touch of the pages
        t0 = time.perf_counter()
        O.grid(p0, none, np.zeros(0, np.complex128), out=self.fw)
        self.t_zero = time.perf_counter() - t0
        # one full-size FFT plane
        pf = type(p).from_buffer_copy(p)
        pf.nf3 = 1
        plane = self.fw[0:1]
        t0 = time.perf_counter()
        O.fft2_planes(pf, plane, +1)
        self.t_fft_plane = time.perf_counter() - t0
        # w stage + corrections per pixel: a 256^2 run minus its gridding and FFT
        small = synth.make("ms2dirty_256_fp64", seed=0, nrow=2000)
        psm = O.setup(small["uvw"], 256, 256, 2.0, 1e8, 1e-5)
        Xs = O.grid_coords(psm, small["uvw"])
        t0 = time.perf_counter()
        O.grid(psm, Xs, small["vis"])
        t_small_grid = time.perf_counter() - t0
        t0 = time.perf_counter()
        O.ms2dirty(small["uvw"], small["vis"], small["wgt"], 256, 256, 2.0, 1e8, 1e-5)
        t1 = time.perf_counter()
        t_small_fft = self.t_fft_plane * (psm.nf1 * psm.nf2) / (p.nf1 * p.nf2) * psm.nf3
        self.t_pix = max((t1 - t0) - t_small_fft - t_small_grid, 0.0) / (256 * 256)

    def sample(self, nsample, seed):
        from cugridder_b200 import synth

        O, p, full = self.O, self.p, self.full
        d = synth.make(self.cfg_name, seed=seed, nrow=nsample)
        ps = type(p).from_buffer_copy(p)
        ps.nrow = nsample
        X = O.grid_coords(ps, d["uvw"])
        c = d["vis"].astype(np.complex128)
        t0 = time.perf_counter()
        O.grid(ps, X, c, out=self.fw)
        t1 = time.perf_counter()
        O.degrid(ps, X, self.fw)
        t2 = time.perf_counter()
        t_grid = max(t1 - t0 - self.t_zero, 0.0) / nsample
        t_degrid = (t2 - t1) / nsample
        M = full["nrow"]
        npix = full["nx"] * full["ny"]
        t_total = (self.t_zero + M * (t_grid + t_degrid) + 2 * p.nf3 * self.t_fft_plane
                   + 2 * npix * self.t_pix)
        return {
            "value": round(M / t_total / 1e6, 6), "unit": "Mvis/s", "cores": O.num_threads(),
            "kind": "port",
            "sample": ("EXTRAPOLATED, not a full run: the oracle (C/OpenMP restatement of the "
                       "reference pipeline) gridded and degridded %d rows (W=%d) on the full "
                       "%dx%dx%d grid, one %dx%d FFT plane per direction x nw=%d, the w stage "
                       "per pixel from a 256^2 run; assembled for %d rows on %dx%d"
                       % (nsample, p.kw, p.nf1, p.nf2, p.nf3, p.nf1, p.nf2, p.nf3, M, full["nx"],
                          full["ny"])),
            "seconds_for_full_workload": round(t_total, 1),
        }


def cpu_reference_rate(cfg_name, nsample=200_000, seed=0):
    return CpuReference(cfg_name).sample(nsample, seed)


def reference_cuda_worker(args):
    """Child process of --impl reference: time the reference's own CUDA build
    (oracle/_ref/libcurafft_ref.so, its sources compiled for sm_100a by
    oracle/ref.mk) through its own host API -- ms2dirty_2 / dirty2ms_2 (FP64
    build) and ms2dirtyf_2 / dirty2msf_2 (FP32 build, FP32 coordinates) -- on
    the main line's data (seed 0).  Its API takes host buffers and returns
    when the result is back, so each call is timed by the host clock; median
    of `reps` calls after one warm-up call.  Prints one JSON line."""
    import ctypes

    from cugridder_b200 import synth

    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libcurafft_ref.so"))
    P, D, F, I = ctypes.c_void_p, ctypes.c_double, ctypes.c_float, ctypes.c_int
    fns = {}
    for name, real in (("ms2dirty_2", D), ("dirty2ms_2", D), ("ms2dirtyf_2", F), ("dirty2msf_2", F)):
        f = getattr(lib, name)
        f.argtypes = [I, I, I, real, real, P, P, P, P, real, real, I]
        f.restype = I
        fns[name] = f
    d = synth.make(args.config, seed=0, nrow=args.nrow)
    img = synth.random_image(d["nx"], d["ny"], seed=1000, dtype=np.complex64)
    M = d["uvw"].shape[0]
    out = {}
    clocks = ClockSampler(0)
    clocks.start()
    for prec in ("fp32", "fp64"):
        single = prec == "fp32"
        rt, ct = (np.float32, np.complex64) if single else (np.float64, np.complex128)
        uvw = np.ascontiguousarray(d["uvw"], dtype=rt)
        vis = np.ascontiguousarray(d["vis"], dtype=ct)
        wgt = np.ascontiguousarray(d["wgt"], dtype=rt)
        dimg = np.ascontiguousarray(img, dtype=ct)
        dirty = np.zeros((d["nx"], d["ny"]), dtype=ct)
        vout = np.zeros(M, dtype=ct)
        sfx = "f" if single else ""
        t_m, t_d, st = [], [], []
        for r in range(args.ref_reps + 1):
            t0 = time.perf_counter()
            s1 = fns["ms2dirty%s_2" % sfx](M, d["nx"], d["ny"], d["fov"], d["freq"], uvw.ctypes.data,
                                           vis.ctypes.data, wgt.ctypes.data, dirty.ctypes.data,
                                           args.eps, 2.0, -1)
            t1 = time.perf_counter()
            s2 = fns["dirty2ms%s_2" % sfx](M, d["nx"], d["ny"], d["fov"], d["freq"], uvw.ctypes.data,
                                           vout.ctypes.data, wgt.ctypes.data, dimg.ctypes.data,
                                           args.eps, 2.0, -1)
            t2 = time.perf_counter()
            st.append([int(s1), int(s2)])
            if r > 0:
                t_m.append(t1 - t0)
                t_d.append(t2 - t1)
        m, dd = statistics.median(t_m), statistics.median(t_d)
        out[prec] = {"value": round(M / (m + dd) / 1e6, 3), "unit": "Mvis/s",
                     "ms2dirty_s": round(m, 4), "dirty2ms_s": round(dd, 4), "reps": args.ref_reps,
                     "status": st[-1],
                     "api": "ms2dirty%s_2 + dirty2ms%s_2 (host buffers)" % (sfx, sfx)}
    clocks.stop()
    out["eps"] = args.eps
    out["timing"] = "host clock around each synchronous call; median after one warm-up call"
    out["clocks"] = clocks.summary()
    print(json.dumps(out), flush=True)


def reference_cuda(args):
    """reference_cuda key of --impl reference (see reference_cuda_worker)."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libcurafft_ref.so")):
        return {"unavailable": "oracle/_ref/libcurafft_ref.so is not built here (build() builds it "
                               "where the reference sources are present)"}
    cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference", "--_ref-cuda-worker",
           "--config", args.config, "--eps", str(args.eps), "--ref-reps", str(args.ref_reps)]
    if args.nrow:
        cmd += ["--nrow", str(args.nrow)]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    except subprocess.TimeoutExpired:
        return {"unavailable": "the reference CUDA build did not finish within 900 s"}
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    if r.returncode != 0 or not lines:
        tail = (r.stderr or r.stdout or "").strip().splitlines()[-1:] or [""]
        return {"unavailable": "the reference CUDA build exited with status %d: %s"
                               % (r.returncode, tail[0][:200])}
    return json.loads(lines[-1])


def run_reference(args, rank, world):
    """--impl reference: rank 0 times the reference algorithm on the host
    cores (the oracle port, extrapolated from samples: CpuReference), and
    reports the reference's own CUDA build beside it (reference_cuda)."""
    if rank != 0:
        return None
    cpu = CpuReference(args.config)
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu.sample(100_000, seed=i)
        if i >= args.warmup:
            vals.append(r)
    del cpu
    v = statistics.median(x["value"] for x in vals)
    r = dict(vals[-1])
    r["value"] = v
    r["reference_cuda"] = reference_cuda(args)
    return r


# --------------------------------------------------------------------------- batched workload
BATCH_METRIC = "Mvis/s batched ms2dirty+dirty2ms, 32 uneven datasets, eps 1e-4, 1 B200"


def make_batch_data(specs, torch):
    """Device arrays of the batched workload, seeded per dataset."""
    out = []
    for sp in specs:
        g = torch.Generator(device="cuda")
        g.manual_seed(sp["seed"])
        n, nc = sp["nrow"], sp["nchan"]
        uv = torch.randn((n, 2), generator=g, device="cuda", dtype=torch.float64) * sp["uv_sigma"]
        uv.clamp_(-sp["uv_clip"], sp["uv_clip"])
        w = (torch.rand((n, 1), generator=g, device="cuda", dtype=torch.float64) * 2 - 1) * sp["w_max"]
        uvw = torch.cat([uv, w], 1).contiguous()
        vis = torch.complex(torch.randn((n, nc), generator=g, device="cuda"),
                            torch.randn((n, nc), generator=g, device="cuda")).contiguous()
        wgt = (torch.rand((n, nc), generator=g, device="cuda") + 0.5).contiguous()
        out.append(dict(uvw=uvw, freqs=sp["freqs"], vis=vis, wgt=wgt, fov=sp["fov"],
                        dirty=torch.zeros((sp["nx"], sp["ny"]), dtype=torch.complex64, device="cuda")))
    return out


def batched_forms(args, kern, steps, warmup, sequential=True):
    """The batched workload (synth.batch_specs: 32 uneven datasets, eps 1e-4)
    through cugridder_b200.batch.Batch -- one persistent spreading /
    interpolation launch per direction, autotuned tiling, CUDA graph replay --
    in three forms: the learned kernel in FP32, ES in FP32 and plain ES in
    FP64; and (sequential=True) the same datasets through one Plan each,
    called in sequence.  One step = ms2dirty then dirty2ms of every dataset;
    Mvis/s = sum(nrow * nchan) / step time.  The visibilities are restored
    between steps, outside the timed brackets."""
    import torch

    from cugridder_b200 import Plan, _lib, synth
    from cugridder_b200.batch import Batch

    eps = 1e-4
    lib = _lib.load()
    specs = synth.batch_specs()
    ds32 = make_batch_data(specs, torch)
    nvis = sum(sp["nrow"] * sp["nchan"] for sp in specs)
    st = torch.cuda.current_stream()

    def timed(step_fn, nsteps, restore):
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(nsteps)]
        torch.cuda.synchronize()
        for k in range(nsteps):
            restore()
            ev[k][0].record(st)
            step_fn(0)
            ev[k][1].record(st)
            step_fn(1)
            ev[k][2].record(st)
        torch.cuda.synchronize()
        m2d = [e[0].elapsed_time(e[1]) for e in ev]
        d2m = [e[1].elapsed_time(e[2]) for e in ev]
        return statistics.median(m2d), statistics.median(d2m)

    es = {"kind": "es", "W": 0, "coef": None}
    out = {}
    clocks = ClockSampler(torch.cuda.current_device())
    for label, kk, prec in (("learned_fp32", kern, "fp32"), ("es_fp32", es, "fp32"),
                            ("es_fp64", es, "fp64")):
        if prec == "fp64":
            ds = [dict(d, vis=d["vis"].to(torch.complex128), wgt=d["wgt"].to(torch.float64),
                       dirty=torch.zeros(d["dirty"].shape, dtype=torch.complex128, device="cuda"))
                  for d in ds32]
        else:
            ds = ds32
        pristine = [d["vis"].clone() for d in ds]

        def restore():
            for d, v in zip(ds, pristine):
                d["vis"].copy_(v)

        b = Batch(ds, epsilon=eps, precision=prec)
        if kk["kind"] == "poly":
            b.set_kernel("poly", kk["W"], kk["coef"])
        l0 = lib.cg_kernel_launches()
        b.ms2dirty()  # eager, autotuned
        b.dirty2ms()
        torch.cuda.synchronize()
        l1 = lib.cg_kernel_launches()
        b.ms2dirty()  # captured
        b.dirty2ms()
        torch.cuda.synchronize()
        launches = lib.cg_kernel_launches() - l1
        for _ in range(max(1, warmup - 2)):
            b.ms2dirty()
            b.dirty2ms()
        if label == "learned_fp32":
            clocks.start()
        m2d, d2m = timed(lambda dr: b.ms2dirty() if dr == 0 else b.dirty2ms(), steps, restore)
        if label == "learned_fp32":
            clocks.stop()
        gt, dt, tms = b.tiling()
        out[label] = {"value": round(nvis / ((m2d + d2m) * 1e-3) / 1e6, 2),
                      "ms_ms2dirty": round(m2d, 3), "ms_dirty2ms": round(d2m, 3),
                      "kernels_per_step": launches, "eager_first_call_launches": l1 - l0,
                      "tiling": {"grid_warp_tile": gt, "degrid_tile": dt,
                                 "phase2_ms": [round(x, 3) for x in tms]},
                      "W": kk["W"] or None}
        restore()
        b.close()
        del b
        if prec == "fp64":
            del ds, pristine
        torch.cuda.synchronize()
        torch.cuda.empty_cache()

    if sequential:
        # the same datasets through one Plan each, called in sequence
        ds = ds32
        seq_m2d = seq_d2m = 0.0
        for d in ds:
            nx, ny = d["dirty"].shape
            p = Plan(nx, ny, d["fov"], eps, precision="fp32")
            if kern["kind"] == "poly":
                p.set_kernel("poly", kern["W"], kern["coef"])
            out_vis = torch.empty_like(d["vis"])

            def step(dr):
                if dr == 0:
                    p.ms2dirty_chan(d["uvw"], d["freqs"], d["vis"], d["wgt"], d["dirty"])
                else:
                    p.dirty2ms_chan(d["uvw"], d["freqs"], d["dirty"], d["wgt"], out_vis)

            step(0)
            step(1)
            m2d, d2m = timed(step, 2, lambda: None)
            seq_m2d += m2d
            seq_d2m += d2m
            p.close()
        out["sequential_plans_learned_fp32"] = {
            "value": round(nvis / ((seq_m2d + seq_d2m) * 1e-3) / 1e6, 2),
            "ms_ms2dirty": round(seq_m2d, 3), "ms_dirty2ms": round(seq_d2m, 3)}
    meta = {"workload": "batch_32_uneven", "datasets": len(specs),
            "rows": sum(sp["nrow"] for sp in specs), "visibilities": nvis,
            "images": sorted({sp["nx"] for sp in specs}), "eps": eps,
            "kernel": kern.get("label", "ES"),
            "l2": "inputs larger than L2 (%.1f GB of visibilities)" % (nvis * 8 / 1e9)}
    del ds32
    torch.cuda.empty_cache()
    return out, meta, clocks.summary()


def run_batch(args):
    """--batch: the batched workload's own line (see batched_forms)."""
    import torch

    args.eps = 1e-4
    torch.cuda.set_device(0)
    kern = select_kernel(args)
    out, meta, clocks = batched_forms(args, kern, args.steps, args.warmup)
    main = out["learned_fp32"]
    line = {"metric": BATCH_METRIC, "value": main["value"], "unit": "Mvis/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(main["ms_ms2dirty"] + main["ms_dirty2ms"], 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (fp64 uvw/coordinates)", "data": "synthetic", "config": meta,
            "forms": out, "clocks": clocks,
            "learned_fp32_over_es_fp64": round(main["value"] / out["es_fp64"]["value"], 3),
            "batched_over_sequential": round(main["value"] / out["sequential_plans_learned_fp32"]["value"], 3)}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.ref_cuda_worker:
        reference_cuda_worker(args)
        return
    if args.batch:
        run_batch(args)
        return
    rank, world, local = dist_setup()
    if args.impl == "reference":
        r = run_reference(args, rank, world)
        if rank == 0:
            line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": "Mvis/s",
                    "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                    "dtype": "f64", "data": "synthetic",
                    "config": workload_config(args, world),
                    "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
                    "e2e": {"value": r["value"], "unit": "Mvis/s", "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 0},
                    "reference_cuda": r["reference_cuda"]}
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    res = run_b200(args, rank, world, local)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_rate(args.config)
    if rank == 0:
        info = res.pop("info")
        line = {
            "metric": METRIC, "value": round(res["value"], 2), "unit": "Mvis/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(res["ms_per_step"], 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (fp64 uvw/coordinates)", "data": "synthetic",
            "config": workload_config(args, world),
            "impl_detail": {"kernel": res["kernel"]["label"], "W": info["kw"], "nw": info["nw"],
                            "grid": [info["nf1"], info["nf2"]],
                            "tiling": dict(res["tiling"], autotuned=not args.no_autotune)},
            "roofline": res["roofline"], "cpu_baseline": cpu, "e2e": res.get("e2e"),
            "gpu_launches": res["gpu_launches"], "clocks": res["clocks"],
            "fp64_plain": res.get("fp64_plain"), "fp32_over_fp64": res.get("fp32_over_fp64"),
            "fp64_eps_leg": res.get("fp64_eps_leg"), "batched": res.get("batched"),
            "accuracy": res.get("accuracy"), "adjointness": res.get("adjointness"),
            "stages": res["stages"],
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
