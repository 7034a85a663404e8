"""Row-split warp tiles of a plan's gridding (k_tile_chunks, the chunk slots of
k_grid_warp, k_split_reduce_plan): a dataset whose rows sit near its grid
centre, so that a few tiles hold most of them.  With CG_SPLIT_ROWS=300 those
tiles run as chunks of at most 300 rows whose partial tiles are summed in
chunk order; the image is checked against the same plan unsplit
(CG_SPLIT=0) and against the oracle, in FP32 and FP64, with the ES and the
learned kernel, for single- and multi-channel calls."""
import numpy as np
import pytest

from cugridder_b200 import Plan, synth
from cugridder_b200.synth import rel_l2

from tests.gpu_helpers import to_dev

pytestmark = pytest.mark.gpu


def _dense(prec, n=64, fov=2.0, nrow=40000, nchan=1, seed=900):
    """Rows concentrated near the grid centre: u, v scaled by 0.05."""
    d = synth.make("ms2dirty_256_fp64", seed=seed, nrow=nrow, nx=n, ny=n, fov=fov)
    uvw = d["uvw"].copy()
    uvw[:, :2] *= 0.05
    cdt, rdt = (np.complex64, np.float32) if prec == "fp32" else (np.complex128, np.float64)
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    vis = (rng.standard_normal((nrow, nchan)) + 1j * rng.standard_normal((nrow, nchan))).astype(cdt)
    wgt = rng.uniform(0.5, 1.5, (nrow, nchan)).astype(rdt)
    freqs = np.linspace(1.0e8, 2.0e8, nchan) if nchan > 1 else np.array([1.0e8])
    return dict(uvw=uvw, vis=vis, wgt=wgt, freqs=freqs, n=n, fov=fov)


def _grid(torch, d, prec, eps, kernel):
    tdt = torch.complex64 if prec == "fp32" else torch.complex128
    p = Plan(d["n"], d["n"], d["fov"], eps, precision=prec)
    if kernel is not None:
        p.set_kernel("poly", kernel.W, kernel.horner)
    out = torch.zeros((d["n"], d["n"]), dtype=tdt, device="cuda")
    p.ms2dirty_chan(to_dev(torch, d["uvw"]), d["freqs"], to_dev(torch, d["vis"]),
                    to_dev(torch, d["wgt"]), out)
    torch.cuda.synchronize()
    p.close()
    return out.cpu().numpy()


def _oracle(d, eps, kernel):
    from oracle import oracle as O

    f0 = d["freqs"][0]
    s = np.array([1.0] + [f / f0 for f in d["freqs"][1:]])
    uvw = (d["uvw"][:, None, :] * s[None, :, None]).reshape(-1, 3)
    if kernel is not None:
        O.set_kernel("poly", kernel.W, kernel.horner)
    try:
        out, _ = O.ms2dirty(uvw, d["vis"].reshape(-1).astype(np.complex128),
                            d["wgt"].reshape(-1).astype(np.float64), d["n"], d["n"], d["fov"], f0, eps)
    finally:
        if kernel is not None:
            O.set_kernel("es")
    return out


@pytest.mark.parametrize("prec,learned,nchan", [("fp32", False, 1), ("fp32", True, 3),
                                                 ("fp64", False, 1), ("fp64", False, 2)])
def test_plan_split_tiles(torch_cuda, monkeypatch, prec, learned, nchan):
    from cugridder_b200.learn import load_kernel

    torch = torch_cuda
    kernel = load_kernel(5) if learned else None
    eps = 1e-4 if prec == "fp32" else 1e-9
    tol_split, tol_oracle = (2e-6, 2e-5) if prec == "fp32" else (1e-13, 1e-10)
    d = _dense(prec, nchan=nchan)
    monkeypatch.setenv("CG_SPLIT", "0")
    whole = _grid(torch, d, prec, eps, kernel)
    monkeypatch.delenv("CG_SPLIT")
    monkeypatch.setenv("CG_SPLIT_ROWS", "300")
    split = _grid(torch, d, prec, eps, kernel)
    again = _grid(torch, d, prec, eps, kernel)
    assert np.array_equal(split, again)  # chunk order fixes the sums: deterministic
    if prec == "fp32":
        assert not np.array_equal(split, whole)  # the chunked sums ran (they round differently)
    assert rel_l2(split, whole) < tol_split
    assert rel_l2(split, _oracle(d, eps, kernel)) < tol_oracle


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_plan_split_tiles_partial_hives(torch_cuda, monkeypatch, prec):
    """Split tiles on a grid whose axes are not multiples of 8 cells (a 42 x 74
    image on a 90 x 150 grid: partial last hives, the exact-wrap kernels), with
    rows over the whole band and aliased past its edge, so that the chunks of
    edge tiles walk wrapped halo hives."""
    from oracle import oracle as O

    torch = torch_cuda
    eps = 1e-4 if prec == "fp32" else 1e-9
    tol_split, tol_oracle = (2e-6, 2e-5) if prec == "fp32" else (1e-13, 1e-10)
    cdt, rdt = (np.complex64, np.float32) if prec == "fp32" else (np.complex128, np.float64)
    tdt = torch.complex64 if prec == "fp32" else torch.complex128
    d = synth.wrap_case(60000, 42, 74, 3.0, freq=1.0e8, seed=950)

    def grid():
        p = Plan(42, 74, 3.0, eps, precision=prec)
        out = torch.zeros((42, 74), dtype=tdt, device="cuda")
        p.ms2dirty(to_dev(torch, d["uvw"]), d["freq"], to_dev(torch, d["vis"].astype(cdt)),
                   to_dev(torch, d["wgt"].astype(rdt)), out)
        torch.cuda.synchronize()
        p.close()
        return out.cpu().numpy()

    monkeypatch.setenv("CG_SPLIT", "0")
    whole = grid()
    monkeypatch.delenv("CG_SPLIT")
    monkeypatch.setenv("CG_SPLIT_ROWS", "300")
    split = grid()
    if prec == "fp32":
        assert not np.array_equal(split, whole)  # the chunked sums ran
    assert rel_l2(split, whole) < tol_split
    ref, _ = O.ms2dirty(d["uvw"], d["vis"].astype(cdt).astype(np.complex128),
                        d["wgt"].astype(rdt).astype(np.float64), 42, 74, 3.0, d["freq"], eps)
    assert rel_l2(split, ref) < tol_oracle
