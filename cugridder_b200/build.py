"""Build libcugridder.so in-tree for sm_100a.

    python -m cugridder_b200.build [--verbose] [--ptxas-info]

Compiles every CUDA source of cugridder_b200/csrc with nvcc
(-gencode arch=compute_100a,code=sm_100a) in parallel and links
cugridder_b200/lib/libcugridder.so, plus libcurafft.so (same library under the
reference's file name, so a reference ctypes binding that loads
"libcurafft.so" finds it).
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libcugridder.so")
ALIAS = os.path.join(LIBDIR, "libcurafft.so")

SOURCES = ["cg_bin.cu", "cg_spread.cu", "cg_grid_slide.cu", "cg_grid_mma.cu", "cg_wstage.cu", "cg_pipeline.cu",
           "cg_capi.cu", "cg_static.cu", "cg_learn.cu",
           "cg_explicit.cu", "cg_fft.cu", "cg_nufft.cu", "cg_batch.cu", "cg_degrid_tma.cu"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def flags(ptxas_info=False):
    f = [
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-O3", "-lineinfo", "-std=c++17",
        "-ccbin", _host_cxx(),
        "-Xcompiler", "-fPIC,-ffp-contract=off,-O3",
        "-I", os.path.join(ROOT, "include"),
    ]
    if ptxas_info:
        f += ["-Xptxas", "-v"]
    return f


def _headers_mtime():
    m = 0.0
    for d in (CSRC, os.path.join(ROOT, "include")):
        for fn in os.listdir(d):
            if fn.endswith((".cuh", ".h", ".hpp")):
                m = max(m, os.path.getmtime(os.path.join(d, fn)))
    return m


def build(verbose=False, ptxas_info=False, force=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = _nvcc()
    hdr = _headers_mtime()
    jobs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        if force or ptxas_info or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr):
            jobs.append([nvcc, "-c", s, "-o", o] + flags(ptxas_info))

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        return cmd, r.returncode, r.stdout

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for cmd, rc, out in ex.map(run, jobs):
            if out and (verbose or ptxas_info or rc):
                sys.stdout.write(out)
            if rc:
                raise RuntimeError("nvcc failed: %s" % cmd[2])
    objs = [os.path.join(OBJ, s.replace(".cu", ".o")) for s in SOURCES]
    if jobs or not os.path.exists(LIB):
        cmd = [nvcc, "-shared", "-o", LIB] + objs + [
            "-gencode", "arch=compute_100a,code=sm_100a", "-ccbin", _host_cxx(),
            "-lcufft", "-Xlinker", "-rpath,/usr/local/cuda/lib64",
        ]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        shutil.copyfile(LIB, ALIAS)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.ptxas_info, a.force))
