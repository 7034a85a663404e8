"""Gridding by x-sliding warp windows (cg_grid_slide.cu) against the oracle's
spreading (the reference's conv_3d_outputdriven_t1, conv.cu:522-627, restated):
every width it covers (W = 4..8, even and odd), FP64 and FP32, the ES and the
learned kernel, band heights 8 / 16 / 32 and segments of 1 to 64 hive columns
(segment starts mid-grid, wrapped warm-up columns at x = 0), rows over the
whole band and past it (periodic wrap on every axis), and end to end."""
import os

import numpy as np
import pytest

from cugridder_b200 import _lib, synth
from cugridder_b200.synth import rel_l2

from tests.gpu_helpers import payload, plan_ms2dirty

pytestmark = pytest.mark.gpu


def _env(env, fn):
    os.environ.update(env)
    try:
        return fn()
    finally:
        for k in env:
            del os.environ[k]


def _grid_vs_oracle(torch, oracle, d, precision, eps, env, kernel=None):
    from cugridder_b200 import Plan

    nx, ny = d["nx"], d["ny"]

    def run():
        cdt = np.complex128 if precision == "fp64" else np.complex64
        rdt = np.float64 if precision == "fp64" else np.float32
        plan = Plan(nx, ny, d["fov"], eps, precision=precision)
        if kernel is not None:
            plan.set_kernel("poly", kernel.W, kernel.horner)
        uvw = torch.from_numpy(d["uvw"]).cuda()
        vis = torch.from_numpy(d["vis"].astype(cdt)).cuda()
        wgt = torch.from_numpy(d["wgt"].astype(rdt)).cuda()
        dirty = torch.zeros((nx, ny), dtype=torch.complex128 if precision == "fp64"
                            else torch.complex64, device="cuda")
        plan.set_stop_stage(2)
        plan.ms2dirty(uvw, d["freq"], vis, wgt, dirty)
        torch.cuda.synchronize()
        return plan

    plan = _env(dict(env, CG_GRID_SLIDE="1"), run)
    if kernel is not None:  # the kernel's width sets the geometry (nw) too
        oracle.set_kernel("poly", kernel.W, kernel.horner)
    try:
        p = oracle.setup(d["uvw"], nx, ny, d["fov"], d["freq"], eps,
                         eps_floor=1.1e-16 if precision == "fp64" else 6e-8)
        ref = oracle.grid(p, oracle.grid_coords(p, d["uvw"]), payload(d, p))
    finally:
        if kernel is not None:
            oracle.set_kernel("es")
    info = plan.info()
    got = plan.copy_buffer(_lib.CG_BUF_GRID)
    plan.close()
    return rel_l2(got, ref), info


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-6)])
@pytest.mark.parametrize("eps", [1e-3, 1e-4, 1e-5, 1e-6, 1e-7])
def test_slide_widths(torch_cuda, oracle, precision, tol, eps):
    """W = 4..8 on the 256^2 case (rows near the grid centre)."""
    d = synth.make("ms2dirty_256_fp64", seed=23, nrow=30000)
    err, info = _grid_vs_oracle(torch_cuda, oracle, d, precision, eps, {})
    assert 4 <= info["kw"] <= 8
    assert err < tol, (info["kw"], err)


@pytest.mark.parametrize("ty", [8, 16, 32])
@pytest.mark.parametrize("seg", [1, 2, 5, 32, 64])
@pytest.mark.parametrize("eps", [1e-5, 1e-6])
def test_slide_shapes_with_wrap(torch_cuda, oracle, ty, seg, eps):
    """Bands of 8/16/32 rows, segments of 1..64 hive columns, rows spread over
    the whole uv band and past it (96 x 160 image: grid 192 x 320, 8-aligned),
    W = 6 and 7, FP64 at 1e-12."""
    d = synth.wrap_case(8000, 96, 160, 3.0, seed=ty * 100 + seg)
    err, info = _grid_vs_oracle(torch_cuda, oracle, d, "fp64", eps,
                                {"CG_SLIDE_TY": str(ty), "CG_SLIDE_SEG": str(seg)})
    assert info["nf1"] % 8 == 0 and info["nf2"] % 8 == 0
    assert err < 1e-12, err


@pytest.mark.parametrize("W", [5, 6, 8])
def test_slide_learned_kernel(torch_cuda, oracle, W):
    from cugridder_b200.learn import available_widths, load_kernel

    if W not in available_widths():
        pytest.skip("no learned kernel of width %d" % W)
    k = load_kernel(W)
    d = synth.wrap_case(20000, 128, 128, 2.0, seed=W)
    err, info = _grid_vs_oracle(torch_cuda, oracle, d, "fp32", 1e-5, {}, kernel=k)
    assert info["kw"] == W
    assert err < 2e-6, err


def test_slide_small_grid_and_warps(torch_cuda, oracle):
    """A 16-cell grid axis (the window's own width) and forced warps per CTA."""
    d = synth.wrap_case(3000, 8, 32, 2.0, seed=5)
    for warps in (1, 3, 16):
        err, info = _grid_vs_oracle(torch_cuda, oracle, d, "fp64", 1e-5,
                                    {"CG_SLIDE_WARPS": str(warps)})
        assert info["nf2"] == 16 or info["nf1"] == 16
        assert err < 1e-12, (warps, err)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 2e-5)])
def test_slide_end_to_end(torch_cuda, oracle, precision, tol):
    d = synth.wrap_case(30000, 128, 96, 3.0, seed=77)
    _, dirty, st = _env({"CG_GRID_SLIDE": "1"},
                        lambda: plan_ms2dirty(torch_cuda, d, precision, 1e-6))
    assert st == 0
    ref, _ = oracle.ms2dirty(d["uvw"], d["vis"], d["wgt"], 128, 96, d["fov"], d["freq"], 1e-6)
    assert rel_l2(dirty, ref) < tol


def test_slide_falls_back_where_it_does_not_apply(torch_cuda, oracle):
    """W = 10 (eps 1e-9) and a grid axis of 250 cells: the tiled kernel runs."""
    d = synth.wrap_case(5000, 122, 96, 3.0, seed=9)
    for eps in (1e-9, 1e-5):
        err, _ = _grid_vs_oracle(torch_cuda, oracle, d, "fp64", eps, {})
        assert err < 1e-12
