"""The shared-memory column FFT (FP32, power-of-two columns) against cuFFT's
strided column transforms, through the whole pipeline in both directions."""
import os

import numpy as np
import pytest

from cugridder_b200 import Plan, synth
from cugridder_b200.synth import rel_l2

from tests.gpu_helpers import to_dev

pytestmark = pytest.mark.gpu


def _narrow_band_case(N, nrow, seed):
    """uv confined to about 30% of the grid rows, so the band-pruned FFT runs."""
    fov = 1.0
    pix = np.deg2rad(fov) / N
    freq = 1.5e8
    u_max = 0.15 / pix * 299792458.0 / freq
    rng = np.random.Generator(np.random.PCG64(seed))
    uvw = np.empty((nrow, 3))
    uvw[:, :2] = rng.uniform(-u_max, u_max, (nrow, 2))
    uvw[:, 2] = rng.uniform(-300.0, 300.0, nrow)
    vis = (rng.standard_normal(nrow) + 1j * rng.standard_normal(nrow)).astype(np.complex64)
    wgt = rng.uniform(0.5, 1.5, nrow).astype(np.float32)
    return dict(uvw=uvw, vis=vis, wgt=wgt, nx=N, ny=N, fov=fov, freq=freq)


def _run(torch, d, img, col_fft):
    os.environ["CG_COL_FFT"] = "1" if col_fft else "0"
    try:
        plan = Plan(d["nx"], d["ny"], d["fov"], 1e-5, precision="fp32")
    finally:
        del os.environ["CG_COL_FFT"]
    uvw = to_dev(torch, d["uvw"], np.float64)
    wgt = to_dev(torch, d["wgt"])
    dirty = torch.zeros((d["nx"], d["ny"]), dtype=torch.complex64, device="cuda")
    plan.ms2dirty(uvw, d["freq"], to_dev(torch, d["vis"]), wgt, dirty)
    vis = torch.zeros(d["uvw"].shape[0], dtype=torch.complex64, device="cuda")
    plan.dirty2ms(uvw, d["freq"], to_dev(torch, img, np.complex64), wgt, vis)
    torch.cuda.synchronize()
    info = plan.info()
    plan.close()
    return dirty.cpu().numpy(), vis.cpu().numpy(), info


VARIANTS = {"registers": {}, "registers_row_kernel": {"CG_ROW_FFT": "1"},
            "registers_pair_exchange": {"CG_COL_FFT_REG": "2"},
            "cluster": {"CG_COL_FFT_REG": "3"}, "four_step": {"CG_COL_FFT_REG": "4"},
            "shared_pair": {"CG_COL_FFT_REG": "0"},
            "shared_single": {"CG_COL_FFT_REG": "0", "CG_COL_FFT_CB": "1"}}


@pytest.mark.parametrize("variant", sorted(VARIANTS))
@pytest.mark.parametrize("N", [512, 1024, 2048, 4096])
def test_column_fft_matches_cufft(torch_cuda, N, variant):
    """Every column kernel: register-resident (default, with the row pass by
    cuFFT or by the register-resident row kernel, with column-pair exchanges,
    or as a four-CTA cluster gathering through distributed shared memory),
    shared-memory resident with two adjacent columns or one column per CTA."""
    d = _narrow_band_case(N, 100_000, seed=N)
    img = synth.random_image(N, N, seed=2)
    env = VARIANTS[variant]
    os.environ.update(env)
    try:
        a = _run(torch_cuda, d, img, True)
    finally:
        for k in env:
            del os.environ[k]
    b = _run(torch_cuda, d, img, False)
    assert a[2]["nf2"] == 2 * N
    assert rel_l2(a[0], b[0]) < 2e-6
    assert rel_l2(a[1], b[1]) < 2e-6


@pytest.mark.parametrize("variant", ["registers", "four_step"])
@pytest.mark.parametrize("nx,ny", [(512, 1024), (1024, 512)])
def test_column_fft_non_square(torch_cuda, nx, ny, variant):
    """Non-square images: the column length (nf2, from nx) and the image rows
    it skips, [nx - nx/2, nf2 - nx/2), differ from the row length (nf1)."""
    d = _narrow_band_case(max(nx, ny), 100_000, seed=nx + 3 * ny)
    d["nx"], d["ny"] = nx, ny
    img = synth.random_image(nx, ny, seed=5)
    env = VARIANTS[variant]
    os.environ.update(env)
    try:
        a = _run(torch_cuda, d, img, True)
    finally:
        for k in env:
            del os.environ[k]
    b = _run(torch_cuda, d, img, False)
    assert a[2]["nf2"] == 2 * nx and a[2]["nf1"] == 2 * ny
    assert rel_l2(a[0], b[0]) < 2e-6
    assert rel_l2(a[1], b[1]) < 2e-6


def test_four_step_16384(torch_cuda):
    """8192 x 8192 image: columns of L = 16384, beyond the one-pass column
    kernels, take the four-step transform by default."""
    d = _narrow_band_case(8192, 200_000, seed=7)
    img = synth.random_image(8192, 8192, seed=8)
    a = _run(torch_cuda, d, img, True)
    b = _run(torch_cuda, d, img, False)
    assert a[2]["nf2"] == 16384
    assert rel_l2(a[0], b[0]) < 2e-6
    assert rel_l2(a[1], b[1]) < 2e-6
