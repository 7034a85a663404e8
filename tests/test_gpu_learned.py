"""Learned kernel on the GPU: the CUDA forward/backward kernels of the MLP
against the oracle's FP64 restatement (the gradient check), the training
primitives (spreading, its adjoint, the FP64 direct sums), the
piecewise-polynomial gridding path against the oracle, and what the trained
kernels gain over ES."""
import numpy as np
import pytest

from cugridder_b200 import Plan, _lib, synth
from cugridder_b200.learn import model as M
from cugridder_b200.synth import rel_l2

from tests.gpu_helpers import to_dev

pytestmark = pytest.mark.gpu


def _theta(seed):
    th = M.init_theta(seed)
    rng = np.random.Generator(np.random.PCG64(seed + 7))
    o = 2 * M.H + M.H * M.H + M.H
    th[o:o + M.H] = rng.normal(0, 0.3, M.H)
    th[-1] = -0.2
    return th


def _stream(torch):
    return torch.cuda.current_stream().cuda_stream


@pytest.mark.parametrize("W", [4, 6, 9])
def test_phi_forward_backward_vs_oracle(torch_cuda, oracle, W):
    torch = torch_cuda
    lib = _lib.load()
    assert lib.cg_learn_theta_size() == M.NTHETA
    th = _theta(W)
    beta0 = M.beta0_for(W)
    rng = np.random.Generator(np.random.PCG64(W))
    n = 20011  # ragged last warp / block
    d = rng.uniform(-W / 2 * 1.05, W / 2 * 1.05, n)  # some points outside the support
    g = rng.normal(size=n)
    th_d = to_dev(torch, th, np.float32)
    d_d = to_dev(torch, d, np.float32)
    phi = torch.empty(n, dtype=torch.float32, device="cuda")
    _lib.check(lib.cg_learn_phi_forward(th_d.data_ptr(), beta0, W, n, d_d.data_ptr(), phi.data_ptr(),
                                        _stream(torch)))
    d32 = d.astype(np.float32).astype(np.float64)
    th32 = th.astype(np.float32).astype(np.float64)
    ref = oracle.learn_phi(th32, beta0, W, d32)
    got = phi.cpu().numpy()
    assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max()
    assert np.all(got[np.abs(d32) >= W / 2] == 0)
    dth = torch.zeros(M.NTHETA, dtype=torch.float32, device="cuda")
    g_d = to_dev(torch, g, np.float32)
    _lib.check(lib.cg_learn_phi_backward(th_d.data_ptr(), beta0, W, n, d_d.data_ptr(), g_d.data_ptr(),
                                         dth.data_ptr(), _stream(torch)))
    ref_g = oracle.learn_phi_grad(th32, beta0, W, d32, g.astype(np.float32).astype(np.float64))
    got_g = dth.cpu().numpy().astype(np.float64)
    # FP32 accumulation over 20k points against FP64
    assert np.linalg.norm(got_g - ref_g) <= 1e-4 * np.linalg.norm(ref_g)


def test_training_spread_and_adjoint(torch_cuda):
    torch = torch_cuda
    lib = _lib.load()
    rng = np.random.Generator(np.random.PCG64(5))
    B, Mv, W, nf = 3, 257, 5, 64
    X = rng.uniform(0, nf, (B, Mv))
    Y = rng.uniform(0, nf, (B, Mv))
    gx0 = (np.floor(X - W / 2) + 1).astype(np.int32)
    gy0 = (np.floor(Y - W / 2) + 1).astype(np.int32)
    phx = rng.uniform(0, 1, (B, Mv, W)).astype(np.float32)
    phy = rng.uniform(0, 1, (B, Mv, W)).astype(np.float32)
    c = rng.normal(size=(B, Mv, 2)).astype(np.float32)
    grid = torch.zeros((B, nf, nf, 2), dtype=torch.float32, device="cuda")
    dev = [to_dev(torch, a) for a in (c, gx0, gy0, phx, phy)]
    _lib.check(lib.cg_learn_spread2d(B, Mv, W, nf, *[t.data_ptr() for t in dev], grid.data_ptr(),
                                     _stream(torch)))
    ref = np.zeros((B, nf, nf, 2))
    for s in range(B):
        for j in range(Mv):
            w = np.outer(phx[s, j], phy[s, j]).astype(np.float64)
            ix = (gx0[s, j] + np.arange(W)) % nf
            iy = (gy0[s, j] + np.arange(W)) % nf
            ref[s][np.ix_(ix, iy)] += w[..., None] * c[s, j]
    np.testing.assert_allclose(grid.cpu().numpy(), ref, rtol=1e-5, atol=1e-5)
    # adjoint: <spread(phx, phy), G> is linear in phx (and in phy) with gradient adj(G)
    G = rng.normal(size=(B, nf, nf, 2)).astype(np.float32)
    G_d = to_dev(torch, G)
    dphx = torch.empty_like(dev[3])
    dphy = torch.empty_like(dev[4])
    _lib.check(lib.cg_learn_spread2d_adjoint(B, Mv, W, nf, *[t.data_ptr() for t in dev],
                                             G_d.data_ptr(), dphx.data_ptr(), dphy.data_ptr(),
                                             _stream(torch)))
    lhs = float((ref * G).sum())
    assert abs(float((dphx.cpu().numpy() * phx).sum()) - lhs) <= 1e-4 * abs(lhs)
    assert abs(float((dphy.cpu().numpy() * phy).sum()) - lhs) <= 1e-4 * abs(lhs)


def test_training_direct_sums(torch_cuda):
    torch = torch_cuda
    lib = _lib.load()
    rng = np.random.Generator(np.random.PCG64(6))
    B, Mv, nf, nk = 2, 500, 128, 37
    X = rng.uniform(0, nf, (B, Mv))
    Y = rng.uniform(0, nf, (B, Mv))
    c = rng.normal(size=(B, Mv, 2))
    k1 = rng.integers(-32, 32, (B, nk)).astype(np.int32)
    k2 = rng.integers(-32, 32, (B, nk)).astype(np.int32)
    F = torch.empty((B, nk, 2), dtype=torch.float64, device="cuda")
    dev = [to_dev(torch, a) for a in (X, Y, c)]
    kd = [to_dev(torch, a) for a in (k1, k2)]
    _lib.check(lib.cg_learn_dft2(B, Mv, nf, dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(),
                                 nk, kd[0].data_ptr(), kd[1].data_ptr(), F.data_ptr(), _stream(torch)))
    cc = c[..., 0] + 1j * c[..., 1]
    ref = np.einsum("sj,skj->sk", cc, np.exp(2j * np.pi * (k1[:, :, None] * X[:, None, :] +
                                                            k2[:, :, None] * Y[:, None, :]) / nf))
    got = F.cpu().numpy()
    np.testing.assert_allclose(got[..., 0] + 1j * got[..., 1], ref, rtol=1e-12, atol=1e-10)


def _poly_plan_run(torch, d, precision, W, coef, direction, img=None):
    cdt = np.complex128 if precision == "fp64" else np.complex64
    rdt = np.float64 if precision == "fp64" else np.float32
    plan = Plan(d["nx"], d["ny"], d["fov"], 1e-5, precision=precision)
    plan.set_kernel("poly", W, coef)
    uvw = to_dev(torch, d["uvw"], np.float64)
    wgt = to_dev(torch, d["wgt"], rdt)
    ctype = torch.complex128 if precision == "fp64" else torch.complex64
    if direction == "ms2dirty":
        vis = to_dev(torch, d["vis"], cdt)
        out = torch.zeros((d["nx"], d["ny"]), dtype=ctype, device="cuda")
        plan.ms2dirty(uvw, d["freq"], vis, wgt, out)
    else:
        dirty = to_dev(torch, img, cdt)
        out = torch.zeros(d["uvw"].shape[0], dtype=ctype, device="cuda")
        plan.dirty2ms(uvw, d["freq"], dirty, wgt, out)
    torch.cuda.synchronize()
    info = plan.info()
    plan.close()
    return out.cpu().numpy(), info


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 2e-5)])
@pytest.mark.parametrize("direction", ["ms2dirty", "dirty2ms"])
def test_poly_kernel_pipeline_vs_oracle(torch_cuda, oracle, precision, tol, direction):
    """A piecewise-polynomial kernel (a random network's Horner fit, W = 5)
    through the GPU pipeline equals the oracle's polynomial-kernel pipeline."""
    torch = torch_cuda
    d = synth.make("ms2dirty_256_fp64", seed=21, nrow=20000, nx=128, ny=96)
    W = 5
    th = _theta(11)
    coef = M.horner_fit(lambda x: M.phi_np(th, M.beta0_for(W), W, x), W)
    img = synth.random_image(128, 96, seed=3)
    got, info = _poly_plan_run(torch, d, precision, W, coef, direction, img)
    assert info["kw"] == W
    oracle.set_kernel("poly", W, coef)
    try:
        if direction == "ms2dirty":
            ref, p = oracle.ms2dirty(d["uvw"], d["vis"], d["wgt"], 128, 96, d["fov"], d["freq"], 1e-5)
        else:
            ref, p = oracle.dirty2ms(d["uvw"], img, d["wgt"], d["fov"], d["freq"], 1e-5)
    finally:
        oracle.set_kernel("es")
    assert (p.kw, p.nf1, p.nf2, p.nf3) == (W, info["nf1"], info["nf2"], info["nw"])
    assert rel_l2(got, ref) < tol


def test_learned_kernels_gain_over_es(torch_cuda, oracle):
    """Each committed learned kernel, run through the full FP32 W-stacking
    pipeline (ms2dirty and dirty2ms), has a smaller error against the FP64
    direct DFT than the ES kernel of the same width."""
    from cugridder_b200.learn import available_widths, load_kernel

    widths = available_widths()
    if not widths:
        pytest.skip("no trained kernels committed")
    torch = torch_cuda
    d = synth.make("wstack_2048_10M", seed=31, nrow=200_000, nx=512, ny=512, fov=2.0)
    img = synth.random_image(512, 512, seed=9)
    rng = np.random.Generator(np.random.PCG64(2))
    pix = rng.choice(512 * 512, 512, replace=False)
    rows = rng.choice(d["uvw"].shape[0], 256, replace=False)
    dft = oracle.dft_ms2dirty(d["uvw"], d["vis"], d["wgt"], 512, 512, d["fov"], d["freq"], pixels=pix)
    dft_v = oracle.dft_dirty2ms(d["uvw"], img, d["wgt"], d["fov"], d["freq"], rows=rows)
    for W in widths:
        k = load_kernel(W)
        errs = {}
        for name, coef in (("learned", k.horner), ("es", M.es_horner(W))):
            dirty, _ = _poly_plan_run(torch, d, "fp32", W, coef, "ms2dirty")
            vis, _ = _poly_plan_run(torch, d, "fp32", W, coef, "dirty2ms", img)
            errs[name] = (rel_l2(dirty.reshape(-1)[pix], dft), rel_l2(vis[rows], dft_v))
        assert errs["learned"][0] < errs["es"][0], (W, errs)
        assert errs["learned"][1] < errs["es"][1], (W, errs)


# ---------------------------------------------------------------- on-device DFT
def test_explicit_dft_vs_oracle(torch_cuda, oracle):
    """The on-device FP64 direct sums equal the oracle's CPU direct DFT
    (pixel subset and full image for ms2dirty, row subset for dirty2ms)."""
    torch = torch_cuda
    lib = _lib.load()
    d = synth.make("ms2dirty_256_fp64", seed=8, nrow=3001, nx=48, ny=40, fov=2.0)
    nx, ny = 48, 40
    img = synth.random_image(nx, ny, seed=4)
    rng = np.random.Generator(np.random.PCG64(9))
    pix = rng.choice(nx * ny, 101, replace=False).astype(np.int64)
    rows = rng.choice(3001, 77, replace=False).astype(np.int64)
    uvw = to_dev(torch, d["uvw"], np.float64)
    vis = to_dev(torch, d["vis"], np.complex128)
    wgt = to_dev(torch, d["wgt"], np.float64)
    dimg = to_dev(torch, img, np.complex128)
    for sign in (-1, 1):
        out = torch.empty(101, dtype=torch.complex128, device="cuda")
        pd = to_dev(torch, pix)
        _lib.check(lib.cg_explicit_ms2dirty(3001, nx, ny, d["fov"], d["freq"], uvw.data_ptr(),
                                            vis.data_ptr(), wgt.data_ptr(), sign, 101, pd.data_ptr(),
                                            out.data_ptr(), _stream(torch)))
        ref = oracle.dft_ms2dirty(d["uvw"], d["vis"], d["wgt"], nx, ny, d["fov"], d["freq"],
                                  sign=sign, pixels=pix)
        assert rel_l2(out.cpu().numpy(), ref) < 1e-12
        full = torch.empty((nx, ny), dtype=torch.complex128, device="cuda")
        _lib.check(lib.cg_explicit_ms2dirty(3001, nx, ny, d["fov"], d["freq"], uvw.data_ptr(),
                                            vis.data_ptr(), None, sign, -1, None, full.data_ptr(),
                                            _stream(torch)))
        ref_full = oracle.dft_ms2dirty(d["uvw"], d["vis"], None, nx, ny, d["fov"], d["freq"], sign=sign)
        assert rel_l2(full.cpu().numpy(), ref_full.reshape(nx, ny)) < 1e-12
        vout = torch.empty(77, dtype=torch.complex128, device="cuda")
        rd = to_dev(torch, rows)
        _lib.check(lib.cg_explicit_dirty2ms(3001, nx, ny, d["fov"], d["freq"], uvw.data_ptr(),
                                            dimg.data_ptr(), wgt.data_ptr(), sign, 77, rd.data_ptr(),
                                            vout.data_ptr(), _stream(torch)))
        ref_v = oracle.dft_dirty2ms(d["uvw"], img, d["wgt"], d["fov"], d["freq"], sign=sign, rows=rows)
        assert rel_l2(vout.cpu().numpy(), ref_v) < 1e-12


def test_es_forced_width_matches_epsilon_choice(torch_cuda):
    """ES forced to the width that epsilon would pick reproduces the default."""
    torch = torch_cuda
    d = synth.make("ms2dirty_256_fp64", seed=12, nrow=5000, nx=64, ny=64)
    outs = []
    for force in (False, True):
        plan = Plan(64, 64, d["fov"], 1e-5, precision="fp64")
        if force:
            plan.set_kernel("es", 6)
        uvw = to_dev(torch, d["uvw"], np.float64)
        vis = to_dev(torch, d["vis"], np.complex128)
        out = torch.zeros((64, 64), dtype=torch.complex128, device="cuda")
        plan.ms2dirty(uvw, d["freq"], vis, None, out)
        torch.cuda.synchronize()
        assert plan.info()["kw"] == 6
        outs.append(out.cpu().numpy())
        plan.close()
    assert np.array_equal(outs[0], outs[1])
