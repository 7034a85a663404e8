"""TMA-staged degridding (k_degrid_tma, FP32, both variants) against the tiled kernel on
the same plans: interior tiles (one bulk tensor copy per tile) and edge
tiles (periodic staging), ES widths 4-8 and the learned kernel.  A second
call reads back the staging error word (a timed-out wait would fail it)."""
import os

import numpy as np
import pytest

from cugridder_b200 import Plan, synth
from cugridder_b200.synth import rel_l2

from tests.gpu_helpers import to_dev

pytestmark = pytest.mark.gpu


def _dirty2ms(torch, d, img, eps, tma, kernel=None, calls=2):
    os.environ["CG_DEGRID_TMA"] = str(int(tma))  # 0: tiled kernel; 1, 2: TMA variants
    try:
        p = Plan(d["nx"], d["ny"], d["fov"], eps, precision="fp32")
    finally:
        del os.environ["CG_DEGRID_TMA"]
    if kernel is not None:
        p.set_kernel("poly", kernel.W, kernel.horner)
    uvw = to_dev(torch, d["uvw"], np.float64)
    wgt = to_dev(torch, d["wgt"], np.float32)
    dimg = to_dev(torch, img, np.complex64)
    outs = []
    for _ in range(calls):
        vis = torch.zeros(d["uvw"].shape[0], dtype=torch.complex64, device="cuda")
        p.dirty2ms(uvw, d["freq"], dimg, wgt, vis)
        torch.cuda.synchronize()
        outs.append(vis.cpu().numpy())
    W = p.info()["kw"]
    p.close()
    return outs, W


@pytest.mark.parametrize("variant", [1, 2, 3, 4])
@pytest.mark.parametrize("N,fov,eps", [(256, 2.0, 1e-3), (512, 1.0, 1e-4), (1024, 3.0, 1e-6)])
def test_tma_degridding_matches_tiled(torch_cuda, N, fov, eps, variant):
    d = synth.make("wstack_2048_10M", seed=N, nrow=200_000, nx=N, ny=N, fov=fov)
    # u, v up to the Nyquist limit, so that rows reach the grid edges too
    umax = 0.45 * N / (2 * np.deg2rad(fov)) * 299792458.0 / d["freq"]
    rng = np.random.Generator(np.random.PCG64(N + 1))
    d["uvw"][:, :2] = rng.uniform(-umax, umax, (d["uvw"].shape[0], 2))
    img = synth.random_image(N, N, seed=N + 2, dtype=np.complex64)
    a, W = _dirty2ms(torch_cuda, d, img, eps, variant)
    b, _ = _dirty2ms(torch_cuda, d, img, eps, 0)
    assert 4 <= W <= 8
    for x in a:
        assert rel_l2(x, b[0]) < 1e-6


@pytest.mark.parametrize("variant", [1, 2, 3])
def test_tma_degridding_learned_kernel(torch_cuda, variant):
    from cugridder_b200.learn import load_kernel

    k = load_kernel(6)
    d = synth.make("wstack_2048_10M", seed=9, nrow=300_000, nx=1024, ny=1024, fov=1.5)
    img = synth.random_image(1024, 1024, seed=10, dtype=np.complex64)
    a, _ = _dirty2ms(torch_cuda, d, img, 1e-5, variant, kernel=k)
    b, _ = _dirty2ms(torch_cuda, d, img, 1e-5, 0, kernel=k)
    for x in a:
        assert rel_l2(x, b[0]) < 1e-6


@pytest.mark.parametrize("nx,ny", [(512, 1024), (1024, 512)])
def test_tma_degridding_non_square(torch_cuda, nx, ny):
    d = synth.make("wstack_2048_10M", seed=nx + ny, nrow=200_000, nx=nx, ny=ny, fov=1.0)
    img = synth.random_image(nx, ny, seed=11, dtype=np.complex64)
    a, _ = _dirty2ms(torch_cuda, d, img, 1e-5, 2)
    b, _ = _dirty2ms(torch_cuda, d, img, 1e-5, 0)
    for x in a:
        assert rel_l2(x, b[0]) < 1e-6
