"""GPU parity tests: the sm_100a path against the oracle (the reference
algorithm restated on the CPU), the FP64 direct DFT, the golden outputs of the
reference's own CUDA build, and adjointness.  All calls go through the C ABI
(plan API on device buffers, or the reference-named host entry points)."""
import numpy as np
import pytest

import cugridder_b200 as cg
from cugridder_b200 import _lib, synth
from cugridder_b200.synth import rel_l2

from tests.gpu_helpers import plan_dirty2ms, plan_ms2dirty

pytestmark = pytest.mark.gpu

# tolerances (relative L2): FP64 vs the oracle's FP64 restatement differs only
# by summation order; FP32 precision-split vs FP64 results is held to eps.
TOL_FP64_ORACLE = 1e-10
EPS_C1 = 1e-5


@pytest.fixture(scope="module")
def c1():
    return synth.make("ms2dirty_256_fp64", seed=0)


@pytest.fixture(scope="module")
def c1_small():
    return synth.make("ms2dirty_256_fp64", seed=11, nrow=20000)


# ---------------------------------------------------------------- binning
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("case", ["c1", "wst", "ny250"])
def test_binning_bit_exact(torch_cuda, oracle, c1, precision, case):
    """Hive offsets (the reference's hive_count), sorted cell keys and the
    permutation are bit-identical to the oracle's restatement of bin_mapping
    (conv_interp_invoker.cu:121-224); the permutation is the stable one."""
    if case == "c1":
        d, nx, ny, eps = c1, 256, 256, 1e-5
    elif case == "wst":
        t = synth.test_wst_case(5000, 32, 128, fov=10, seed=3)
        d = dict(uvw=t["uvw"], vis=t["ms"], wgt=t["wgt"], fov=10.0, freq=1e9)
        nx, ny, eps = 32, 128, 5e-5
    else:
        t = synth.test_wst_case(3000, 64, 250, fov=20, seed=4)
        d = dict(uvw=t["uvw"], vis=t["ms"], wgt=t["wgt"], fov=20.0, freq=1e9)
        nx, ny, eps = 64, 250, 1e-5
    plan, _, st = plan_ms2dirty(torch_cuda, d, precision, eps, stop=1, nx=nx, ny=ny)
    assert st == 0
    p = oracle.setup(d["uvw"], nx, ny, d["fov"], d["freq"], eps,
                     eps_floor=1.1e-16 if precision == "fp64" else 6e-8)
    info = plan.info()
    assert (info["kw"], info["nf1"], info["nf2"], info["nw"]) == (p.kw, p.nf1, p.nf2, p.nf3)
    assert info["gamma"] == p.gamma and info["i_center"] == p.i_center
    hs_o, perm_o = oracle.bin_mapping(p, d["uvw"])
    keys_o = oracle.bin_keys(p, d["uvw"])
    hs = plan.copy_buffer(_lib.CG_BUF_HIVE_START)
    perm = plan.copy_buffer(_lib.CG_BUF_PERM)
    keys = plan.copy_buffer(_lib.CG_BUF_SORTED_KEYS)
    assert np.array_equal(hs.astype(np.int64), hs_o)
    assert np.array_equal(perm, perm_o)
    assert np.array_equal(keys, keys_o[perm_o])


def test_binning_large_random(torch_cuda, oracle):
    """3.2M rows (782 radix tiles, ragged last tile) stay bit-exact."""
    d = synth.make("wstack_2048_10M", seed=5, nrow=3_200_123)
    plan, _, st = plan_ms2dirty(torch_cuda, d, "fp32", 1e-5, stop=1)
    p = oracle.setup(d["uvw"], d["nx"], d["ny"], d["fov"], d["freq"], 1e-5, eps_floor=6e-8)
    keys_o = oracle.bin_keys(p, d["uvw"])
    perm = plan.copy_buffer(_lib.CG_BUF_PERM)
    assert np.array_equal(perm, np.argsort(keys_o, kind="stable"))
    hs = plan.copy_buffer(_lib.CG_BUF_HIVE_START).astype(np.int64)
    nh = p.nhive[0] * p.nhive[1] * p.nhive[2]
    assert np.array_equal(hs, np.concatenate([[0], np.cumsum(np.bincount(keys_o // 64, minlength=nh))]))


# ---------------------------------------------------------------- kernel tables
def test_fseries_tables(torch_cuda, oracle, c1_small):
    plan, _, _ = plan_ms2dirty(torch_cuda, c1_small, "fp64", EPS_C1)
    p = oracle.setup(c1_small["uvw"], 256, 256, 2.0, 1e8, EPS_C1)
    assert rel_l2(plan.copy_buffer(_lib.CG_BUF_FSERIES_1), oracle.fseries_uv(p, p.nf1)) < 1e-14
    assert rel_l2(plan.copy_buffer(_lib.CG_BUF_FSERIES_2), oracle.fseries_uv(p, p.nf2)) < 1e-14
    k3, _ = oracle.fseries_w(p)
    assert rel_l2(plan.copy_buffer(_lib.CG_BUF_FSERIES_W), k3) < 1e-13


# ---------------------------------------------------------------- gridding stage
def _payload(d, p, sign=-1):
    """c_j = vis * wgt * exp(i o_c w_eff) (ra_exec.cu:103-111; cuft.cu:46-66)."""
    w_eff = (d["uvw"][:, 2] * (d["freq"] / synth.C_LIGHT * sign)) * (2 * np.pi)
    c = d["vis"].astype(np.complex128) * d["wgt"].astype(np.float64)
    return c * np.exp(1j * p.o_center * w_eff)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-6)])
def test_grid_vs_oracle(torch_cuda, oracle, c1_small, precision, tol):
    plan, _, _ = plan_ms2dirty(torch_cuda, c1_small, precision, EPS_C1, stop=2)
    p = oracle.setup(c1_small["uvw"], 256, 256, 2.0, 1e8, EPS_C1)
    X = oracle.grid_coords(p, c1_small["uvw"])
    ref = oracle.grid(p, X, _payload(c1_small, p))
    assert rel_l2(plan.copy_buffer(_lib.CG_BUF_GRID), ref) < tol


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-6)])
def test_degrid_vs_oracle(torch_cuda, oracle, c1_small, precision, tol):
    img = synth.random_image(256, 256, seed=2)
    plan, vis, _ = plan_dirty2ms(torch_cuda, c1_small, img, precision, EPS_C1, stop=0)
    p = oracle.setup(c1_small["uvw"], 256, 256, 2.0, 1e8, EPS_C1)
    ref, _ = oracle.dirty2ms(c1_small["uvw"], img, c1_small["wgt"], 2.0, 1e8, EPS_C1)
    assert rel_l2(vis, ref) < (1e-10 if precision == "fp64" else EPS_C1)


# ---------------------------------------------------------------- end to end
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_ms2dirty_c1(torch_cuda, oracle, c1, precision):
    """256x256, fov 2 deg, 100k rows, eps 1e-5: oracle, DFT subset."""
    _, dirty, st = plan_ms2dirty(torch_cuda, c1, precision, EPS_C1)
    assert st == 0
    ref, _ = oracle.ms2dirty(c1["uvw"], c1["vis"], c1["wgt"], 256, 256, 2.0, 1e8, EPS_C1)
    assert rel_l2(dirty, ref) < (TOL_FP64_ORACLE if precision == "fp64" else EPS_C1)
    pix = np.random.default_rng(0).choice(256 * 256, 512, replace=False)
    dft = oracle.dft_ms2dirty(c1["uvw"], c1["vis"], c1["wgt"], 256, 256, 2.0, 1e8, pixels=pix)
    assert rel_l2(dirty.reshape(-1)[pix], dft) < 2 * EPS_C1


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_dirty2ms_c1(torch_cuda, oracle, c1, precision):
    img = synth.random_image(256, 256, seed=1)
    _, vis, st = plan_dirty2ms(torch_cuda, c1, img, precision, EPS_C1)
    assert st == 0
    ref, _ = oracle.dirty2ms(c1["uvw"], img, c1["wgt"], 2.0, 1e8, EPS_C1)
    assert rel_l2(vis, ref) < (TOL_FP64_ORACLE if precision == "fp64" else EPS_C1)
    rows = np.arange(0, 100_000, 500)
    dft = oracle.dft_dirty2ms(c1["uvw"], img, c1["wgt"], 2.0, 1e8, rows=rows)
    assert rel_l2(vis[rows], dft) < 2 * EPS_C1


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-6)])
def test_adjointness_c1(torch_cuda, c1, precision, tol):
    """<dirty2ms(d), v> = <d, ms2dirty(v)> (complex inner products)."""
    img = synth.random_image(256, 256, seed=4).astype(np.complex128)
    img.imag = np.random.default_rng(9).standard_normal(img.shape)
    _, dirty, _ = plan_ms2dirty(torch_cuda, c1, precision, EPS_C1)
    _, vis, _ = plan_dirty2ms(torch_cuda, c1, img, precision, EPS_C1)
    v = c1["vis"].astype(np.complex128)
    lhs = np.vdot(vis.astype(np.complex128), v)
    rhs = np.vdot(img, dirty.astype(np.complex128))
    assert abs(lhs - rhs) <= tol * abs(rhs)


# ---------------------------------------------------------------- reference API
WST = [(n, nx, ny, fov, eps) for n in (2, 27, 100) for (nx, ny) in ((32, 128), (64, 250), (16, 64))
       for fov in (1, 10, 20) for eps in (2e-1, 5e-3, 5e-5, 5e-7, 5e-12)]


@pytest.mark.parametrize("use_wgt", [False, True])
@pytest.mark.parametrize("single", [False, True])
def test_reference_pytest_matrix(torch_cuda, oracle, single, use_wgt):
    """The reference's own pytest matrix (test_wst.py:36-95) through the
    NIFTY-style binding: adjointness at rtol 1e-12 (FP64) / 5e-5 (FP32), and --
    what the reference only prints -- the error against the FP64 DFT, held to
    the oracle's own error (+ eps)."""
    for (nrow, nx, ny, fov, eps) in WST:
        if single and eps < 5e-6:
            continue
        t = synth.test_wst_case(nrow, nx, ny, fov, single=single, use_wgt=use_wgt)
        xpix, ypix = fov * np.pi / 180 / nx, fov * np.pi / 180 / ny
        freq = np.array([t["freq"]])
        dirty2 = cg.ms2dirty(t["uvw"], freq, t["ms"], t["wgt"], nx, ny, xpix, ypix, 0, 0, eps,
                             True).astype("f8")
        ms2 = cg.dirty2ms(t["uvw"], freq, t["dirty"], t["wgt"], xpix, ypix, 0, 0, eps,
                          True).astype("c16")
        tol = 5e-5 if single else 1e-12
        a, b = np.vdot(t["ms"], ms2[:, 0]).real, np.vdot(dirty2, t["dirty"])
        assert abs(a - b) <= tol * abs(b), (nrow, nx, ny, fov, eps)
        w64 = None if t["wgt"] is None else t["wgt"].astype(np.float64)
        truth = oracle.dft_ms2dirty(t["uvw"], t["ms"], w64, nx, ny, fov, t["freq"]).real
        own, _ = oracle.ms2dirty(t["uvw"], t["ms"], w64, nx, ny, fov, t["freq"], eps)
        bound = rel_l2(own.real, truth) + (eps if not single else max(eps, 2e-6))
        assert rel_l2(dirty2, truth) <= bound, (nrow, nx, ny, fov, eps)


def test_reference_api_sign_plus(torch_cuda, oracle):
    """curagridder.vis2dirty / dirty2vis (sign = +1)."""
    t = synth.test_wst_case(1000, 64, 64, fov=5, seed=7, use_wgt=False)
    dirty = np.zeros((64, 64), np.complex128)
    cg.vis2dirty(t["uvw"], [1e9], t["ms"], None, dirty, 5.0, 1e-7)
    ref, _ = oracle.ms2dirty(t["uvw"], t["ms"], None, 64, 64, 5, 1e9, 1e-7, sign=1)
    assert rel_l2(dirty, ref) < 1e-10
    img = np.zeros((64, 64), np.complex128)
    img.real = t["dirty"]
    ms = np.zeros(1000, np.complex128)
    cg.dirty2vis(t["uvw"], [1e9], ms, None, img, 5.0, 1e-7)
    ref, _ = oracle.dirty2ms(t["uvw"], img, None, 5, 1e9, 1e-7, sign=1)
    assert rel_l2(ms, ref) < 1e-10


def test_mixed_host_api(torch_cuda, oracle, c1):
    d = cg.ms2dirty_mixed(c1["uvw"], 1e8, c1["vis"].astype(np.complex64),
                          c1["wgt"].astype(np.float32), 256, 256, 2.0, EPS_C1)
    ref, _ = oracle.ms2dirty(c1["uvw"], c1["vis"], c1["wgt"], 256, 256, 2.0, 1e8, EPS_C1)
    assert rel_l2(d, ref) < EPS_C1
    img = synth.random_image(256, 256, seed=1)
    v = cg.dirty2ms_mixed(c1["uvw"], 1e8, img.astype(np.complex64), c1["wgt"].astype(np.float32),
                          2.0, EPS_C1)
    ref, _ = oracle.dirty2ms(c1["uvw"], img, c1["wgt"], 2.0, 1e8, EPS_C1)
    assert rel_l2(v, ref) < EPS_C1


# ---------------------------------------------------------------- golden (reference build)
def test_against_reference_build(torch_cuda, golden, c1):
    """Outputs of the reference's own CUDA build on the same inputs."""
    img = synth.random_image(256, 256, seed=1)
    dirty = np.zeros((256, 256), np.complex128)
    assert cg.ms2dirty_2(100000, 256, 256, 2.0, 1e8, c1["uvw"], c1["vis"], c1["wgt"], dirty, 1e-5,
                         2.0, -1) == 0
    assert rel_l2(dirty, golden["c1_fp64/dirty"]) < TOL_FP64_ORACLE
    vis = np.zeros(100000, np.complex128)
    assert cg.dirty2ms_2(100000, 256, 256, 2.0, 1e8, c1["uvw"], vis, c1["wgt"], img, 1e-5, 2.0,
                         -1) == 0
    g = golden["c1_fp64/vis"]
    assert rel_l2(vis[: g.size], g) < TOL_FP64_ORACLE
    # FP32 twins: within 2 eps of the reference's FP32 build (whose own error
    # against FP64 is part of the budget)
    dirty32 = np.zeros((256, 256), np.complex64)
    assert cg.ms2dirtyf_2(100000, 256, 256, 2.0, 1e8, c1["uvw"].astype(np.float32),
                          c1["vis"].astype(np.complex64), c1["wgt"].astype(np.float32), dirty32,
                          1e-5, 2.0, -1) == 0
    assert rel_l2(dirty32, golden["c1_fp32/dirty"]) < 2 * EPS_C1 + rel_l2(golden["c1_fp32/dirty"],
                                                                         golden["c1_fp64/dirty"])


# ---------------------------------------------------------------- edge cases
def test_edge_cases(torch_cuda, oracle):
    t = synth.test_wst_case(50, 32, 32, fov=4, seed=8)
    # empty input: zero image, nothing to write
    d = np.ones((32, 32), np.complex128)
    assert cg.ms2dirty_1(0, 32, 32, 4.0, 1e9, np.zeros((0, 3)), np.zeros(0, complex), d, 1e-6,
                         2.0, -1) == 0
    assert not d.any()
    # a single row
    one = dict(uvw=t["uvw"][:1], vis=t["ms"][:1], wgt=None, fov=4.0, freq=1e9)
    _, img, _ = plan_ms2dirty(torch_cuda, one, "fp64", 1e-9, nx=32, ny=32, use_wgt=False)
    ref, _ = oracle.ms2dirty(one["uvw"], one["vis"], None, 32, 32, 4, 1e9, 1e-9)
    assert rel_l2(img, ref) < 1e-10
    # all rows at the same w (w range of zero width)
    flat = dict(uvw=t["uvw"].copy(), vis=t["ms"], wgt=t["wgt"], fov=4.0, freq=1e9)
    flat["uvw"][:, 2] = 0.03
    _, img, _ = plan_ms2dirty(torch_cuda, flat, "fp64", 1e-9, nx=32, ny=32)
    ref, _ = oracle.ms2dirty(flat["uvw"], flat["vis"], flat["wgt"], 32, 32, 4, 1e9, 1e-9)
    assert rel_l2(img, ref) < 1e-10
    # epsilon below the floor: clipped, status 1, still correct
    dd = np.zeros((32, 32), np.complex128)
    assert cg.ms2dirty_2(50, 32, 32, 4.0, 1e9, t["uvw"], t["ms"], t["wgt"], dd, 1e-30, 2.0, -1) == 1
    ref, _ = oracle.ms2dirty(t["uvw"], t["ms"], t["wgt"], 32, 32, 4, 1e9, 1e-30)
    assert rel_l2(dd, ref) < 1e-10
    # odd image size and non-finite coordinates are rejected with status 2
    assert cg.ms2dirty_1(50, 31, 32, 4.0, 1e9, t["uvw"], t["ms"], np.zeros((31, 32), complex),
                         1e-6, 2.0, -1) == 2
    bad = t["uvw"].copy()
    bad[7, 1] = np.nan
    assert cg.ms2dirty_1(50, 32, 32, 4.0, 1e9, bad, t["ms"], np.zeros((32, 32), complex), 1e-6,
                         2.0, -1) == 2
    # non-default sigma
    for sig in (1.5, 2.5):
        d2 = np.zeros((32, 32), np.complex128)
        assert cg.ms2dirty_2(50, 32, 32, 4.0, 1e9, t["uvw"], t["ms"], t["wgt"], d2, 1e-7, sig,
                             -1) == 0
        ref, _ = oracle.ms2dirty(t["uvw"], t["ms"], t["wgt"], 32, 32, 4, 1e9, 1e-7, sigma=sig)
        assert rel_l2(d2, ref) < 1e-10


def test_determinism(torch_cuda, c1_small):
    """Stable binning + fixed kernel order: two FP64 runs agree bit for bit in
    the binning; images agree to rounding of the atomic accumulation order."""
    p1, a, _ = plan_ms2dirty(torch_cuda, c1_small, "fp64", EPS_C1, stop=1)
    p2, b, _ = plan_ms2dirty(torch_cuda, c1_small, "fp64", EPS_C1, stop=1)
    assert np.array_equal(p1.copy_buffer(_lib.CG_BUF_PERM), p2.copy_buffer(_lib.CG_BUF_PERM))


# ---------------------------------------------------------------- tiled kernels
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-6)])
@pytest.mark.parametrize("method", [0, 1, 2])
def test_grid_methods(torch_cuda, oracle, c1_small, precision, tol, method):
    """Direct (global atomics), warp-tiled (shared memory) and tensor-core
    (3xTF32 hive GEMM, FP32 only; FP64 falls back to the tiled kernel)
    gridding all match the oracle's spreading of the same payload."""
    import os

    os.environ["CG_GRID_METHOD"] = str(method)
    try:
        plan, _, _ = plan_ms2dirty(torch_cuda, c1_small, precision, EPS_C1, stop=2)
    finally:
        del os.environ["CG_GRID_METHOD"]
    p = oracle.setup(c1_small["uvw"], 256, 256, 2.0, 1e8, EPS_C1)
    ref = oracle.grid(p, oracle.grid_coords(p, c1_small["uvw"]), _payload(c1_small, p))
    assert rel_l2(plan.copy_buffer(_lib.CG_BUF_GRID), ref) < tol


@pytest.mark.parametrize("shape", [(8, 16, 3), (16, 8, 5), (24, 40, 1), (32, 32, 0)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_tile_shapes(torch_cuda, oracle, precision, shape):
    """Forced tile shapes and plane batches (partial edge tiles, plane halos
    across batches, batches wrapping around the w axis) give the oracle's
    results in both directions."""
    import os

    t = synth.test_wst_case(4000, 64, 250, fov=20, seed=13)
    d = dict(uvw=t["uvw"], vis=t["ms"], wgt=t["wgt"], fov=20.0, freq=1e9)
    tx, ty, pb = shape
    env = {"CG_TILE_X": str(tx), "CG_TILE_Y": str(ty), "CG_TILE_PLANES": str(pb)}
    os.environ.update(env)
    try:
        _, img, _ = plan_ms2dirty(torch_cuda, d, precision, 1e-6, nx=64, ny=250)
        im = synth.random_image(64, 250, seed=3)
        _, vis, _ = plan_dirty2ms(torch_cuda, d, im, precision, 1e-6)
    finally:
        for k in env:
            del os.environ[k]
    tol = 1e-10 if precision == "fp64" else 2e-5
    ref, _ = oracle.ms2dirty(d["uvw"], d["vis"], d["wgt"], 64, 250, 20, 1e9, 1e-6)
    assert rel_l2(img, ref) < tol
    ref, _ = oracle.dirty2ms(d["uvw"], im, d["wgt"], 20, 1e9, 1e-6)
    assert rel_l2(vis, ref) < tol


@pytest.mark.parametrize("eps", [1e-2, 1e-5, 1e-9])
def test_grid_smaller_than_a_tile(torch_cuda, oracle, eps):
    """8 x 12 image: the upsampled grid is smaller than one 32 x 32 tile, so
    hives are reached through both periodic wraps at once."""
    t = synth.test_wst_case(500, 8, 12, fov=2, seed=21)
    d = dict(uvw=t["uvw"], vis=t["ms"], wgt=t["wgt"], fov=2.0, freq=1e9)
    _, img, _ = plan_ms2dirty(torch_cuda, d, "fp64", eps, nx=8, ny=12)
    ref, _ = oracle.ms2dirty(d["uvw"], d["vis"], d["wgt"], 8, 12, 2, 1e9, eps)
    assert rel_l2(img, ref) < 1e-10
    im = synth.random_image(8, 12, seed=5)
    _, vis, _ = plan_dirty2ms(torch_cuda, d, im, "fp64", eps)
    ref, _ = oracle.dirty2ms(d["uvw"], im, d["wgt"], 2, 1e9, eps)
    assert rel_l2(vis, ref) < 1e-10


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("fp32", 1e-6)])
def test_fft_band_pruning(torch_cuda, c1, precision, tol):
    """The band-pruned separable FFT (rows of the data band, columns of the
    image) gives the full 2-D transform's results in both directions."""
    import os

    img = synth.random_image(256, 256, seed=6)
    out = {}
    for prune in ("1", "0"):
        os.environ["CG_FFT_PRUNE"] = prune
        try:
            _, d, _ = plan_ms2dirty(torch_cuda, c1, precision, EPS_C1)
            _, v, _ = plan_dirty2ms(torch_cuda, c1, img, precision, EPS_C1)
        finally:
            del os.environ["CG_FFT_PRUNE"]
        out[prune] = (d, v)
    assert rel_l2(out["1"][0], out["0"][0]) < tol
    assert rel_l2(out["1"][1], out["0"][1]) < tol


@pytest.mark.parametrize("eps", [5e-3, 1e-4, 1e-5, 1e-6, 1e-7])
def test_tensor_core_gridding_widths(torch_cuda, oracle, eps):
    """Tensor-core gridding for every kernel width it covers (W = 4..8, even
    and odd), including sparse hives below the GEMM threshold, against the
    oracle's spreading."""
    import os

    d = synth.make("ms2dirty_256_fp64", seed=17, nrow=30000)
    os.environ["CG_GRID_METHOD"] = "2"
    try:
        plan, _, _ = plan_ms2dirty(torch_cuda, d, "fp32", eps, stop=2)
    finally:
        del os.environ["CG_GRID_METHOD"]
    p = oracle.setup(d["uvw"], 256, 256, 2.0, 1e8, eps, eps_floor=6e-8)
    ref = oracle.grid(p, oracle.grid_coords(p, d["uvw"]), _payload(d, p))
    assert rel_l2(plan.copy_buffer(_lib.CG_BUF_GRID), ref) < 2e-6
