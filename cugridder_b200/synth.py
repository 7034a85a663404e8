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


def wrap_case(nrow, nx, ny, fov, freq=1.0e9, seed=0, reach=1.2, w_frac=0.1):
    """Rows spread over the WHOLE uv grid and past its edge: u and v uniform in
    +-reach times the image's Nyquist limit (1 / (2 pixel size) wavelengths),
    so after the shift to [0, nf) rows land in every cell, including the first
    and last hive of each axis, and with reach > 1 alias around the periodic
    wrap.  w ~ U(-w_frac, w_frac) times the u limit.  vis complex N(0, 1),
    wgt U(0.5, 1.5)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    rad = np.deg2rad(fov)
    lam = C_LIGHT / freq
    umax = reach * nx / (2.0 * rad) * lam  # metres
    vmax = reach * ny / (2.0 * rad) * lam
    uvw = np.empty((nrow, 3), dtype=np.float64)
    uvw[:, 0] = rng.uniform(-umax, umax, nrow)
    uvw[:, 1] = rng.uniform(-vmax, vmax, nrow)
    uvw[:, 2] = rng.uniform(-w_frac * umax, w_frac * umax, nrow)
    vis = rng.standard_normal(nrow) + 1j * rng.standard_normal(nrow)
    wgt = rng.uniform(0.5, 1.5, nrow)
    return dict(uvw=uvw, vis=vis, wgt=wgt, nx=nx, ny=ny, fov=float(fov), freq=float(freq))


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


# Batched uneven solves: 32 independent datasets with row counts log-uniform
# in [1e4, 1e7], images from {512, 1024, 2048}, fov U(1, 4) deg and 1-16
# channels spaced uniformly in [1e8, 2e8] Hz sharing one uvw set; epsilon
# 1e-4.  u, v, w follow the 4096 case (u, v ~ N(0, 0.3 clip) clipped to
# +-clip, w ~ U(-clip/10, clip/10)) scaled so that the clip sits at the same
# fraction of each image's Nyquist limit at the highest frequency as the 4096
# case's 20 km does at 1.5e8 Hz (10000 wavelengths of 4096 / (2 * 5 deg)).
BATCH_NYQUIST_FRACTION = 10000.0 / (4096 / (2 * np.deg2rad(5.0)))


def batch_specs(n=32, seed=2024, rows_lo=1e4, rows_hi=1e7, sizes=(512, 1024, 2048)):
    """Per-dataset parameters of the batched workload (no arrays)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(n):
        nrow = int(round(10 ** rng.uniform(np.log10(rows_lo), np.log10(rows_hi))))
        size = int(rng.choice(sizes))
        fov = float(rng.uniform(1.0, 4.0))
        nchan = int(rng.integers(1, 17))
        freqs = np.linspace(1.0e8, 2.0e8, nchan) if nchan > 1 else np.array([1.5e8])
        nyq = size / (2 * np.deg2rad(fov))  # wavelengths
        clip = BATCH_NYQUIST_FRACTION * nyq * C_LIGHT / freqs.max()  # metres
        out.append(dict(nrow=nrow, nx=size, ny=size, fov=fov, nchan=nchan, freqs=freqs,
                        uv_clip=clip, uv_sigma=0.3 * clip, w_max=0.1 * clip, seed=seed * 1000 + i))
    return out
