"""Periodic wrap coverage: rows spread over the whole uv grid and past its
edge (synth.wrap_case), on grids whose size is not a multiple of the 8-cell
hive (nf % 8 in {2, 4, 6}: the last hive of an axis is partial).

A row in the first cells of an axis reaches the last cells through the
periodic wrap and vice versa (the reference's conv_3d_outputdriven_t1 wraps
every tap, conv.cu:591-618, and interp_3d_nputsdriven likewise,
interp.cu:132-210).  Every gridding method, forced tile shapes and both
directions end to end are compared with the oracle's restatement."""
import os

import numpy as np
import pytest

from cugridder_b200 import _lib, synth
from cugridder_b200.synth import rel_l2

from tests.gpu_helpers import payload, plan_dirty2ms, plan_ms2dirty

# (nx, ny): nf = next235beven(2 n) gives 90 / 150 (nf % 8 = 2 / 6), 250 / 500
# (2 / 4) and 54 / 270 (6 / 6)
SHAPES = [(42, 74), (122, 250), (26, 132)]


def _case(nx, ny, seed, nrow=6000, fov=3.0):
    return synth.wrap_case(nrow, nx, ny, fov, seed=seed)


def _with_env(env, fn):
    os.environ.update(env)
    try:
        return fn()
    finally:
        for k in env:
            del os.environ[k]


def test_wrap_fixture_reaches_every_edge_hive(oracle):
    """The fixture's rows occupy the first and the last (partial) hive of
    both grid axes, and some alias past the band edge."""
    for i, (nx, ny) in enumerate(SHAPES):
        d = _case(nx, ny, seed=i)
        p = oracle.setup(d["uvw"], nx, ny, d["fov"], d["freq"], 1e-6)
        assert p.nf1 % 8 != 0 or p.nf2 % 8 != 0
        keys = oracle.bin_keys(p, d["uvw"])
        h = keys // 64
        hx, hy = h % p.nhive[0], (h // p.nhive[0]) % p.nhive[1]
        assert {0, p.nhive[0] - 1} <= set(np.unique(hx).tolist())
        assert {0, p.nhive[1] - 1} <= set(np.unique(hy).tolist())
        u_nyq = nx / (2 * np.deg2rad(d["fov"])) * synth.C_LIGHT / d["freq"]
        assert (np.abs(d["uvw"][:, 0]) > u_nyq).any()


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-6)])
@pytest.mark.parametrize("method", [0, 1, 2])
@pytest.mark.parametrize("eps", [1e-5, 1e-6])
@pytest.mark.parametrize("shape", SHAPES)
def test_wrap_gridding_all_methods(torch_cuda, oracle, shape, eps, method, precision, tol):
    """Direct, warp-tiled and tensor-core gridding (FP64 falls back to the
    warp tiles for method 2) at W = 6 and 7 against the oracle's spreading."""
    nx, ny = shape
    d = _case(nx, ny, seed=nx + ny)
    plan, _, st = _with_env({"CG_GRID_METHOD": str(method)},
                            lambda: plan_ms2dirty(torch_cuda, d, precision, eps, stop=2))
    assert st == 0
    p = oracle.setup(d["uvw"], nx, ny, d["fov"], d["freq"], eps,
                     eps_floor=1.1e-16 if precision == "fp64" else 6e-8)
    ref = oracle.grid(p, oracle.grid_coords(p, d["uvw"]), payload(d, p))
    assert rel_l2(plan.copy_buffer(_lib.CG_BUF_GRID), ref) < tol


@pytest.mark.gpu
@pytest.mark.parametrize("wtile", [(16, 8, 3), (16, 16, 0), (32, 24, 5), (16, 8, 64)])
@pytest.mark.parametrize("eps", [1e-5, 1e-6, 1e-9])
@pytest.mark.parametrize("shape", SHAPES)
def test_wrap_warp_tile_shapes(torch_cuda, oracle, shape, eps, wtile):
    """Forced warp-tile shapes and plane batches (64 = all planes) at W = 6,
    7 and 10: tiles at both edges of both axes take their halo rows from the
    partial last hive and from hive 0."""
    nx, ny = shape
    d = _case(nx, ny, seed=3 * nx + ny)
    env = {"CG_WTILE_X": str(wtile[0]), "CG_WTILE_Y": str(wtile[1]),
           "CG_WTILE_PLANES": str(wtile[2])}
    plan, _, st = _with_env(env, lambda: plan_ms2dirty(torch_cuda, d, "fp64", eps, stop=2))
    assert st == 0
    p = oracle.setup(d["uvw"], nx, ny, d["fov"], d["freq"], eps)
    ref = oracle.grid(p, oracle.grid_coords(p, d["uvw"]), payload(d, p))
    assert rel_l2(plan.copy_buffer(_lib.CG_BUF_GRID), ref) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(8, 16, 3), (16, 8, 5), (24, 40, 1), (32, 32, 0)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_wrap_degrid_tile_shapes(torch_cuda, oracle, precision, shape):
    """Forced degridding tile shapes and plane batches: tiles at the grid
    edges stage their halo across the periodic wrap (FP32 runs the tiled
    kernel here, as the forced shape asks)."""
    tx, ty, pb = shape
    d = _case(122, 250, seed=17)
    img = synth.random_image(122, 250, seed=4)
    env = {"CG_TILE_X": str(tx), "CG_TILE_Y": str(ty), "CG_TILE_PLANES": str(pb),
           "CG_DEGRID_TMA": "0"}
    _, vis, st = _with_env(env, lambda: plan_dirty2ms(torch_cuda, d, img, precision, 1e-6))
    assert st == 0
    ref, _ = oracle.dirty2ms(d["uvw"], img, d["wgt"], d["fov"], d["freq"], 1e-6)
    assert rel_l2(vis, ref) < (1e-10 if precision == "fp64" else 2e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("tma", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("shape", SHAPES)
def test_wrap_end_to_end(torch_cuda, oracle, shape, tma):
    """ms2dirty and dirty2ms, FP64 and the FP32 precision split, against the
    oracle; FP32 degridding by the tiled kernel (0) and every TMA variant."""
    nx, ny = shape
    d = _case(nx, ny, seed=5 * nx + ny, nrow=20000)
    img = synth.random_image(nx, ny, seed=nx)
    eps = 1e-6
    ref_d, _ = oracle.ms2dirty(d["uvw"], d["vis"], d["wgt"], nx, ny, d["fov"], d["freq"], eps)
    ref_v, _ = oracle.dirty2ms(d["uvw"], img, d["wgt"], d["fov"], d["freq"], eps)
    for precision, tol in (("fp64", 1e-10), ("fp32", 2e-5)):
        if precision == "fp64" and tma:
            continue
        _, dirty, st = plan_ms2dirty(torch_cuda, d, precision, eps)
        assert st == 0
        assert rel_l2(dirty, ref_d) < tol
        _, vis, st = _with_env({"CG_DEGRID_TMA": str(tma)},
                               lambda: plan_dirty2ms(torch_cuda, d, img, precision, eps))
        assert st == 0
        assert rel_l2(vis, ref_v) < tol
