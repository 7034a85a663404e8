"""Batched solves (cg_batch_*) against the oracle and against one plan per
dataset: uneven datasets (image sizes, fov, rows, channels, one without rows,
one non-square image on a grid with partial last hives and rows over its
whole band), the eager and autotuned first call, the captured second call and
graph replays with new visibilities / images; and the untuned eager form.

The oracle sees each dataset as the library defines multi-channel calls:
row r of channel c becomes row r * nchan + c at f_0 = freqs[0] with
uvw * (f_c / f_0), which has the same phase as row r at f_c.  A direct sum
over the channels at their own frequencies checks that definition itself."""
import numpy as np
import pytest

from cugridder_b200 import Plan, synth
from cugridder_b200.batch import Batch
from cugridder_b200.synth import rel_l2

from tests.gpu_helpers import to_dev

pytestmark = pytest.mark.gpu

# (nx, ny, fov, rows, channels); the 42 x 74 image (grid 90 x 150) has rows
# over its whole band and past it
SPECS = [(64, 64, 1.0, 3000, 1), (96, 96, 2.5, 12000, 3), (128, 128, 1.5, 20000, 2),
         (64, 64, 4.0, 5000, 4), (80, 80, 3.0, 800, 1), (128, 128, 2.0, 30000, 1),
         (64, 64, 2.0, 0, 2), (42, 74, 3.0, 6000, 2)]


def _datasets(torch):
    out = []
    for i, (nx, ny, fov, nrow, nchan) in enumerate(SPECS):
        if nx == ny:
            d = synth.make("ms2dirty_256_fp64", seed=100 + i, nrow=nrow, nx=nx, ny=ny, fov=fov)
        else:
            d = synth.wrap_case(nrow, nx, ny, fov, freq=1.0e8, seed=100 + i)
        freqs = np.linspace(1.0e8, 2.0e8, nchan) if nchan > 1 else np.array([1.0e8])
        rng = np.random.Generator(np.random.PCG64(200 + i))
        vis = (rng.standard_normal((nrow, nchan)) + 1j * rng.standard_normal((nrow, nchan))).astype(np.complex64)
        wgt = rng.uniform(0.5, 1.5, (nrow, nchan)).astype(np.float32)
        out.append(dict(uvw=to_dev(torch, d["uvw"]), freqs=freqs, vis=to_dev(torch, vis),
                        wgt=to_dev(torch, wgt), fov=fov, h_uvw=d["uvw"], h_wgt=wgt, h_vis=vis,
                        dirty=torch.zeros((nx, ny), dtype=torch.complex64, device="cuda")))
    return out


def _flatten(d):
    """The dataset's rows and channels as the library flattens them."""
    f0 = d["freqs"][0]
    s = np.array([1.0] + [f / f0 for f in d["freqs"][1:]])
    uvw = (d["h_uvw"][:, None, :] * s[None, :, None]).reshape(-1, 3)
    return uvw, f0


def _oracle_ref(d, direction, eps, kernel=None):
    """The oracle's result for one dataset of the batch (channels flattened)."""
    from oracle import oracle as O

    nx, ny = d["dirty"].shape
    uvw, f0 = _flatten(d)
    wgt = d["h_wgt"].reshape(-1).astype(np.float64)
    if kernel is not None:
        O.set_kernel("poly", kernel.W, kernel.horner)
    try:
        if direction == 0:
            vis = d["vis"].cpu().numpy().reshape(-1)
            out, _ = O.ms2dirty(uvw, vis, wgt, nx, ny, d["fov"], f0, eps)
        else:
            out, _ = O.dirty2ms(uvw, d["dirty"].cpu().numpy(), wgt, d["fov"], f0, eps)
            out = out.reshape(d["vis"].shape)
    finally:
        if kernel is not None:
            O.set_kernel("es")
    return out


def _close_oracle(out, d, direction, eps, kernel=None, tol=2e-5):
    ref = _oracle_ref(d, direction, eps, kernel)
    if ref.size == 0 or not np.any(ref):
        return not np.any(out)
    return rel_l2(out, ref) < tol


def _plan_ref(torch, d, direction, kernel=None):
    nx, ny = d["dirty"].shape
    p = Plan(nx, ny, d["fov"], 1e-4, precision="fp32")
    if kernel is not None:
        p.set_kernel("poly", kernel.W, kernel.horner)
    if direction == 0:
        out = torch.zeros_like(d["dirty"])
        p.ms2dirty_chan(d["uvw"], d["freqs"], d["vis"], d["wgt"], out)
    else:
        out = torch.zeros_like(d["vis"])
        p.dirty2ms_chan(d["uvw"], d["freqs"], d["dirty"], d["wgt"], out)
    torch.cuda.synchronize()
    p.close()
    return out.cpu().numpy()


def _close(out, ref):
    if ref.size == 0 or not np.any(ref):  # a dataset without rows: an exactly zero result
        return not np.any(out)
    return rel_l2(out, ref) < 1e-5


def _check_batch(torch, ds, b, ncalls, kernel=None):
    for call in range(ncalls):
        for i, d in enumerate(ds):
            d["vis"].mul_(complex(0.5 + 0.1 * call, 0.2))
        b.ms2dirty()
        torch.cuda.synchronize()
        for i, d in enumerate(ds):
            out = d["dirty"].cpu().numpy()
            assert _close(out, _plan_ref(torch, d, 0, kernel)), call
            assert _close_oracle(out, d, 0, 1e-4, kernel), (call, i)
    for call in range(ncalls):
        for i, d in enumerate(ds):
            d["dirty"].copy_(torch.from_numpy(
                synth.random_image(d["dirty"].shape[0], d["dirty"].shape[1], seed=500 + 10 * call + i,
                                   dtype=np.complex64)).cuda())
        b.dirty2ms()
        torch.cuda.synchronize()
        for i, d in enumerate(ds):
            out = d["vis"].cpu().numpy()
            assert _close(out, _plan_ref(torch, d, 1, kernel)), call
            assert _close_oracle(out, d, 1, 1e-4, kernel), (call, i)


def test_batch_learned_kernel(torch_cuda):
    from cugridder_b200.learn import load_kernel

    torch = torch_cuda
    k = load_kernel(5)
    ds = _datasets(torch)
    b = Batch(ds, epsilon=1e-4, precision="fp32")
    b.set_kernel("poly", k.W, k.horner)
    _check_batch(torch, ds, b, 3, kernel=k)
    b.close()


@pytest.mark.parametrize("learned", [False, True])
def test_batch_sliding_windows(torch_cuda, monkeypatch, learned):
    """Every dataset gridded by x-sliding windows in the one launch
    (k_grid_slide_multi: per-dataset band and segment items, window shapes
    and geometry), through the eager, captured and replayed calls, against
    one plan per dataset and the oracle.  Only the datasets whose grids the
    sliding kernel takes (both axes multiples of 8 cells)."""
    from cugridder_b200.learn import load_kernel

    torch = torch_cuda
    monkeypatch.setenv("CG_GRID_SLIDE", "1")
    monkeypatch.setenv("CG_BATCH_AUTOTUNE", "0")
    ds = [d for d, spec in zip(_datasets(torch), SPECS) if spec[0] == spec[1]]
    k = load_kernel(5) if learned else None
    b = Batch(ds, epsilon=1e-4, precision="fp32")
    if k is not None:
        b.set_kernel("poly", k.W, k.horner)
    _check_batch(torch, ds, b, 3, kernel=k)
    b.close()


def test_batch_untuned_eager(torch_cuda, monkeypatch):
    torch = torch_cuda
    monkeypatch.setenv("CG_BATCH_AUTOTUNE", "0")
    monkeypatch.setenv("CG_BATCH_GRAPH", "0")
    ds = _datasets(torch)
    b = Batch(ds, epsilon=1e-4, precision="fp32")
    _check_batch(torch, ds, b, 2)
    assert b.tiling()[0] == (0, 0, 0, 0) and b.tiling()[1] == (0, 0, 0, 0)
    b.close()


def test_batch_matches_plans_through_graph_replays(torch_cuda):
    torch = torch_cuda
    ds = _datasets(torch)
    b = Batch(ds, epsilon=1e-4, precision="fp32")
    for call in range(4):  # eager (autotuned), captured, replay, replay
        for i, d in enumerate(ds):  # new visibilities every call, same tensors
            d["vis"].mul_(complex(0.5 + 0.1 * call, 0.2))
        b.ms2dirty()
        torch.cuda.synchronize()
        for d in ds:
            assert _close(d["dirty"].cpu().numpy(), _plan_ref(torch, d, 0)), call
            assert _close_oracle(d["dirty"].cpu().numpy(), d, 0, 1e-4), call
    for call in range(3):
        for i, d in enumerate(ds):
            d["dirty"].copy_(torch.from_numpy(
                synth.random_image(d["dirty"].shape[0], d["dirty"].shape[1], seed=300 + 10 * call + i,
                                   dtype=np.complex64)).cuda())
        b.dirty2ms()
        torch.cuda.synchronize()
        for d in ds:
            assert _close(d["vis"].cpu().numpy(), _plan_ref(torch, d, 1)), call
            assert _close_oracle(d["vis"].cpu().numpy(), d, 1, 1e-4), call
    grid_t, degrid_t, ms = b.tiling()
    assert grid_t[0] in (16, 32) and grid_t[1] in (8, 16, 32), grid_t
    assert degrid_t[3] in (256, 512), degrid_t
    assert ms[0] > 0 and ms[1] > 0, ms
    b.close()


def test_batch_fp64_matches_plans(torch_cuda):
    """FP64 batch (the double instantiations of the one-launch kernels)
    against one FP64 plan per dataset."""
    torch = torch_cuda
    ds = []
    for i, (n, _, fov, nrow, nchan) in enumerate(SPECS[:4]):
        d = synth.make("ms2dirty_256_fp64", seed=400 + i, nrow=nrow, nx=n, ny=n, fov=fov)
        freqs = np.linspace(1.0e8, 2.0e8, nchan) if nchan > 1 else np.array([1.0e8])
        rng = np.random.Generator(np.random.PCG64(500 + i))
        vis = rng.standard_normal((nrow, nchan)) + 1j * rng.standard_normal((nrow, nchan))
        wgt = rng.uniform(0.5, 1.5, (nrow, nchan))
        ds.append(dict(uvw=to_dev(torch, d["uvw"]), freqs=freqs, vis=to_dev(torch, vis),
                       wgt=to_dev(torch, wgt), fov=fov, h_uvw=d["uvw"], h_wgt=wgt,
                       dirty=torch.zeros((n, n), dtype=torch.complex128, device="cuda")))
    b = Batch(ds, epsilon=1e-9, precision="fp64")
    for call in range(3):
        b.ms2dirty()
        torch.cuda.synchronize()
        for d in ds:
            n = d["dirty"].shape[0]
            p = Plan(n, n, d["fov"], 1e-9, precision="fp64")
            out = torch.zeros_like(d["dirty"])
            p.ms2dirty_chan(d["uvw"], d["freqs"], d["vis"], d["wgt"], out)
            torch.cuda.synchronize()
            p.close()
            assert rel_l2(d["dirty"].cpu().numpy(), out.cpu().numpy()) < 1e-12, call
            assert _close_oracle(d["dirty"].cpu().numpy(), d, 0, 1e-9, tol=1e-10), call
    for call in range(2):
        b.dirty2ms()
        torch.cuda.synchronize()
        for d in ds:
            n = d["dirty"].shape[0]
            p = Plan(n, n, d["fov"], 1e-9, precision="fp64")
            out = torch.zeros_like(d["vis"])
            p.dirty2ms_chan(d["uvw"], d["freqs"], d["dirty"], d["wgt"], out)
            torch.cuda.synchronize()
            p.close()
            assert rel_l2(d["vis"].cpu().numpy(), out.cpu().numpy()) < 1e-12, call
            assert _close_oracle(d["vis"].cpu().numpy(), d, 1, 1e-9, tol=1e-10), call
    b.close()


def test_batch_channel_flattening_vs_direct_sums(torch_cuda):
    """The flattened-channel definition itself: the batch's image equals the
    FP64 direct sum over every (row, channel) at the channel's own frequency,
    and its visibilities the direct adjoint sums per channel, within 2 eps on
    pixel / row subsets."""
    from oracle import oracle as O

    torch = torch_cuda
    ds = _datasets(torch)
    b = Batch(ds, epsilon=1e-4, precision="fp32")
    b.ms2dirty()
    torch.cuda.synchronize()
    images = [d["dirty"].cpu().numpy() for d in ds]
    imgs_in = []
    for i, d in enumerate(ds):
        img = synth.random_image(d["dirty"].shape[0], d["dirty"].shape[1], seed=700 + i,
                                 dtype=np.complex64)
        imgs_in.append(img)
        d["dirty"].copy_(torch.from_numpy(img).cuda())
    b.dirty2ms()
    torch.cuda.synchronize()
    rng = np.random.default_rng(5)
    for i, d in enumerate(ds):
        nx, ny = images[i].shape
        nrow, nchan = d["vis"].shape
        if nrow == 0:
            continue
        vis_out = d["vis"].cpu().numpy()  # dirty2ms output; the ms2dirty input is h_vis
        wgt = d["h_wgt"].astype(np.float64)
        pix = rng.choice(nx * ny, min(256, nx * ny), replace=False)
        rows = rng.choice(nrow, min(256, nrow), replace=False)
        for c in range(nchan):
            truth_v = O.dft_dirty2ms(d["h_uvw"], imgs_in[i], wgt[:, c], d["fov"], d["freqs"][c],
                                     rows=rows)
            assert rel_l2(vis_out[rows, c], truth_v) < 2e-4, (i, c)
        truth_d = sum(O.dft_ms2dirty(d["h_uvw"], d["h_vis"][:, c], wgt[:, c], nx, ny, d["fov"],
                                     d["freqs"][c], pixels=pix) for c in range(nchan))
        assert rel_l2(images[i].reshape(-1)[pix], truth_d) < 2e-4, i
    b.close()


def _split_datasets(torch, prec):
    """Square datasets of SPECS plus one whose rows sit near its grid centre
    (u, v scaled by 0.05: most rows in a few tiles), in precision prec."""
    cdt, rdt = (np.complex64, np.float32) if prec == "fp32" else (np.complex128, np.float64)
    tdt = torch.complex64 if prec == "fp32" else torch.complex128
    specs = [s for s in SPECS if s[0] == s[1] and s[3] > 0] + [(64, 64, 2.0, 40000, 2)]
    out = []
    for i, (n, _, fov, nrow, nchan) in enumerate(specs):
        d = synth.make("ms2dirty_256_fp64", seed=600 + i, nrow=nrow, nx=n, ny=n, fov=fov)
        uvw = d["uvw"].copy()
        if i == len(specs) - 1:
            uvw[:, :2] *= 0.05
        freqs = np.linspace(1.0e8, 2.0e8, nchan) if nchan > 1 else np.array([1.0e8])
        rng = np.random.Generator(np.random.PCG64(700 + i))
        vis = (rng.standard_normal((nrow, nchan)) + 1j * rng.standard_normal((nrow, nchan))).astype(cdt)
        wgt = rng.uniform(0.5, 1.5, (nrow, nchan)).astype(rdt)
        out.append(dict(uvw=to_dev(torch, uvw), freqs=freqs, vis=to_dev(torch, vis),
                        wgt=to_dev(torch, wgt), fov=fov, h_uvw=uvw, h_wgt=wgt, h_vis=vis,
                        dirty=torch.zeros((n, n), dtype=tdt, device="cuda")))
    return out


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_batch_split_tiles(torch_cuda, monkeypatch, prec):
    """Heavy warp tiles gridded as row chunks into partial tiles summed in
    chunk order (CG_BATCH_SPLIT_ROWS=300: chunks of at most 300 rows, so the
    dense dataset's central tiles split many ways) against the same batch
    unsplit (CG_BATCH_SPLIT=0), one plan per dataset and the oracle, through
    the eager, captured and replayed calls.  The captured call launches one
    kernel more than the unsplit one: the reduce pass."""
    from cugridder_b200 import _lib

    torch = torch_cuda
    lib = _lib.load()
    eps, tol_split, tol_oracle = (1e-4, 2e-6, 2e-5) if prec == "fp32" else (1e-9, 1e-13, 1e-10)
    ds = _split_datasets(torch, prec)

    def run(env, ncalls):
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        b = Batch(ds, epsilon=eps, precision=prec)
        outs, launches = [], []
        for call in range(ncalls):  # eager (autotuned, split plan), captured, replayed
            l0 = lib.cg_kernel_launches()
            b.ms2dirty()
            torch.cuda.synchronize()
            launches.append(lib.cg_kernel_launches() - l0)
            outs.append([d["dirty"].cpu().numpy().copy() for d in ds])
        tiling = b.tiling()
        b.close()
        for k in env:
            monkeypatch.delenv(k)
        return outs, launches, tiling

    ref, ref_launches, ref_tiling = run({"CG_BATCH_SPLIT": "0", "CG_BATCH_AUTOTUNE": "0"}, 2)
    outs, launches, tiling = run({"CG_BATCH_SPLIT_ROWS": "300", "CG_BATCH_AUTOTUNE": "0"}, 3)
    assert tiling[0] == ref_tiling[0]
    assert launches[1] == ref_launches[1] + 1, (launches, ref_launches)
    for call in range(3):
        for i, d in enumerate(ds):
            assert rel_l2(outs[call][i], ref[0][i]) < tol_split, (call, i)
    for i, d in enumerate(ds):
        assert _close_oracle(outs[2][i], d, 0, eps, tol=tol_oracle), i
        if prec == "fp32":
            assert _close(outs[2][i], _plan_ref(torch, d, 0)), i
