"""Seeded synthetic visibility sets with the shapes and distributions of the
benchmark configurations (no public dataset is involved; the configurations
define their inputs completely).

Each generator returns a dict with uvw [nrow,3] float64 (metres), vis,
wgt, and the imaging parameters.  numpy's PCG64 Generator is used so the
streams are reproducible across numpy versions.
"""
import numpy as np

C_LIGHT = 299792458.0

CONFIGS = {
    # 256x256, fov 2 deg, 100k rows at 1e8 Hz, FP64 vis, eps 1e-5
    "ms2dirty_256_fp64": dict(nx=256, ny=256, fov=2.0, nrow=100_000, freq=1.0e8, uv_sigma=1500.0,
                              uv_clip=5000.0, w_max=200.0, cplx=np.complex128, real=np.float64,
                              eps=1e-5),
    # 4096x4096, fov 5 deg, 20M rows at 1.5e8 Hz, complex64 vis, float32 wgt
    "wstack_4096_20M": dict(nx=4096, ny=4096, fov=5.0, nrow=20_000_000, freq=1.5e8,
                            uv_sigma=6000.0, uv_clip=20000.0, w_max=2000.0, cplx=np.complex64,
                            real=np.float32, eps=1e-5),
    # 2048x2048, fov 3 deg, 10M rows (evaluation set of the kernel study)
    "wstack_2048_10M": dict(nx=2048, ny=2048, fov=3.0, nrow=10_000_000, freq=1.5e8,
                            uv_sigma=4000.0, uv_clip=16000.0, w_max=1000.0, cplx=np.complex64,
                            real=np.float32, eps=1e-5),
    # 8192x8192, fov 6 deg, 200M rows at 1.2e8 Hz
    "wstack_8192_200M": dict(nx=8192, ny=8192, fov=6.0, nrow=200_000_000, freq=1.2e8,
                             uv_sigma=10000.0, uv_clip=40000.0, w_max=4000.0, cplx=np.complex64,
                             real=np.float32, eps=1e-6),
}


def make(name=None, seed=0, nrow=None, **over):
    """Dataset for a named configuration (optionally overriding fields)."""
    cfg = dict(CONFIGS[name]) if name else {}
    cfg.update(over)
    if nrow is not None:
        cfg["nrow"] = int(nrow)
    rng = np.random.Generator(np.random.PCG64(seed))
    n = cfg["nrow"]
    uv = rng.normal(0.0, cfg["uv_sigma"], size=(n, 2))
    np.clip(uv, -cfg["uv_clip"], cfg["uv_clip"], out=uv)
    w = rng.uniform(-cfg["w_max"], cfg["w_max"], size=n)
    uvw = np.empty((n, 3), dtype=np.float64)
    uvw[:, :2] = uv
    uvw[:, 2] = w
    del uv, w
    cplx = cfg.get("cplx", np.complex128)
    real = cfg.get("real", np.float64)
    vis = np.empty(n, dtype=cplx)
    vis.real = rng.standard_normal(n, dtype=np.float64 if real == np.float64 else np.float32)
    vis.imag = rng.standard_normal(n, dtype=np.float64 if real == np.float64 else np.float32)
    wgt = rng.uniform(0.5, 1.5, size=n).astype(real)
    out = dict(cfg)
    out.update(uvw=uvw, vis=vis, wgt=wgt, seed=seed)
    return out


def test_wst_case(nrow, nxdirty, nydirty, fov, seed=42, f0=1e9, use_wgt=True, single=False):
    """Inputs shaped like the reference's pytest cases (test_wst.py:59-66):
    uvw = (rand-0.5)/(f0/c), ms and dirty uniform in [-0.5, 0.5)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    uvw = (rng.random((nrow, 3)) - 0.5) / (f0 / C_LIGHT)
    ms = rng.random(nrow) - 0.5 + 1j * (rng.random(nrow) - 0.5)
    dirty = rng.random((nxdirty, nydirty)) - 0.5
    wgt = rng.random(nrow) if use_wgt else None
    if single:
        ms = ms.astype(np.complex64)
        dirty = dirty.astype(np.float32)
        if wgt is not None:
            wgt = wgt.astype(np.float32)
    return dict(uvw=uvw, ms=ms, dirty=dirty, wgt=wgt, freq=f0, fov=fov, nx=nxdirty, ny=nydirty)


def random_image(nx, ny, seed=1, dtype=np.complex128):
    rng = np.random.Generator(np.random.PCG64(seed))
    img = np.zeros((nx, ny), dtype=dtype)
    img.real = rng.standard_normal((nx, ny))
    return img


def rel_l2(a, b):
    """||a - b|| / ||b|| (b is the reference)."""
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2) / np.sum(np.abs(b) ** 2)))
