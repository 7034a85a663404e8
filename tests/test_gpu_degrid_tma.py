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


@pytest.mark.parametrize("variant", [1, 2])
def test_tma_stage_wait_timeout_is_reported_by_the_call(torch_cuda, variant):
    """A staging wait that runs out fails THAT call with CG_ERR_CUDA.

    CG_TMA_STAGE_WAIT_TRIES=0 (a test-only bound) makes the wait for every
    CTA's first staged box give up at once; the CTA stops taking tiles, and
    the drain of its boxes still in flight keeps the full bound, so no copy
    is pending when it exits.  The plan API and the host API both return the
    error from the call that hit it; the next call on the same plan is clean
    and correct, and cg_plan_status then reports nothing."""
    from cugridder_b200 import _lib, dirty2ms_mixed, release_cache

    N = 1024
    d = synth.make("wstack_2048_10M", seed=77, nrow=200_000, nx=N, ny=N, fov=1.0)
    img = synth.random_image(N, N, seed=78, dtype=np.complex64)
    ref, _ = _dirty2ms(torch_cuda, d, img, 1e-5, 0, calls=1)
    os.environ["CG_DEGRID_TMA"] = str(variant)
    try:
        p = Plan(N, N, d["fov"], 1e-5, precision="fp32")
    finally:
        del os.environ["CG_DEGRID_TMA"]
    uvw = to_dev(torch_cuda, d["uvw"], np.float64)
    wgt = to_dev(torch_cuda, d["wgt"], np.float32)
    dimg = to_dev(torch_cuda, img, np.complex64)
    vis = torch_cuda.zeros(d["uvw"].shape[0], dtype=torch_cuda.complex64, device="cuda")
    os.environ["CG_TMA_STAGE_WAIT_TRIES"] = "0"
    try:
        with pytest.raises(_lib.GridderError) as ex:
            p.dirty2ms(uvw, d["freq"], dimg, wgt, vis)
    finally:
        del os.environ["CG_TMA_STAGE_WAIT_TRIES"]
    assert ex.value.code == 3 and "timed out" in str(ex.value)
    vis.zero_()
    assert p.dirty2ms(uvw, d["freq"], dimg, wgt, vis) == 0
    torch_cuda.cuda.synchronize()
    assert rel_l2(vis.cpu().numpy(), ref[0]) < 1e-6
    assert p.check_status() == 0
    p.close()
    # host-pointer API (its cached plan runs the default TMA variant 2)
    if variant == 2:
        release_cache()
        os.environ["CG_TMA_STAGE_WAIT_TRIES"] = "0"
        try:
            with pytest.raises(_lib.GridderError) as ex:
                dirty2ms_mixed(d["uvw"], d["freq"], img, d["wgt"], d["fov"], 1e-5)
        finally:
            del os.environ["CG_TMA_STAGE_WAIT_TRIES"]
        assert ex.value.code == 3
        v = dirty2ms_mixed(d["uvw"], d["freq"], img, d["wgt"], d["fov"], 1e-5)
        assert rel_l2(v, ref[0]) < 1e-6
