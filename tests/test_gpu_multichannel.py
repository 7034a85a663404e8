"""Multi-channel calls (cg_plan_ms2dirty_chan / cg_plan_dirty2ms_chan) against
the FP64 direct DFT summed over channels, adjointness, and the single-channel
identity."""
import numpy as np
import pytest

from cugridder_b200 import GridderError, Plan, synth
from cugridder_b200.synth import rel_l2

from tests.gpu_helpers import to_dev

pytestmark = pytest.mark.gpu

FREQS = [1.0e8, 1.31e8, 1.77e8]


def _data(nchan, seed=3, nrow=6000):
    d = synth.make("ms2dirty_256_fp64", seed=seed, nrow=nrow, nx=96, ny=80, fov=2.0)
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    vis = rng.standard_normal((nrow, nchan)) + 1j * rng.standard_normal((nrow, nchan))
    wgt = rng.uniform(0.5, 1.5, (nrow, nchan))
    return d, vis, wgt


@pytest.mark.parametrize("precision,eps", [("fp64", 1e-7), ("fp32", 1e-5)])
def test_multichannel_vs_dft(torch_cuda, oracle, precision, eps):
    torch = torch_cuda
    d, vis, wgt = _data(len(FREQS))
    cdt = np.complex128 if precision == "fp64" else np.complex64
    rdt = np.float64 if precision == "fp64" else np.float32
    tc = torch.complex128 if precision == "fp64" else torch.complex64
    plan = Plan(96, 80, d["fov"], eps, precision=precision)
    uvw = to_dev(torch, d["uvw"], np.float64)
    dirty = torch.zeros((96, 80), dtype=tc, device="cuda")
    plan.ms2dirty_chan(uvw, FREQS, to_dev(torch, vis, cdt), to_dev(torch, wgt, rdt), dirty)
    img = synth.random_image(96, 80, seed=5)
    vout = torch.zeros((d["uvw"].shape[0], len(FREQS)), dtype=tc, device="cuda")
    plan.dirty2ms_chan(uvw, FREQS, to_dev(torch, img, cdt), to_dev(torch, wgt, rdt), vout)
    torch.cuda.synchronize()
    plan.close()
    ref = sum(oracle.dft_ms2dirty(d["uvw"], vis[:, c], wgt[:, c], 96, 80, d["fov"], f)
              for c, f in enumerate(FREQS))
    assert rel_l2(dirty.cpu().numpy(), ref) < 2 * eps
    rows = np.arange(0, d["uvw"].shape[0], 17)
    v = vout.cpu().numpy()
    for c, f in enumerate(FREQS):
        rv = oracle.dft_dirty2ms(d["uvw"], img, wgt[:, c], d["fov"], f, rows=rows)
        assert rel_l2(v[rows, c], rv) < 2 * eps


def test_multichannel_adjoint(torch_cuda):
    torch = torch_cuda
    d, vis, wgt = _data(len(FREQS), seed=7)
    plan = Plan(96, 80, d["fov"], 1e-9, precision="fp64")
    uvw = to_dev(torch, d["uvw"], np.float64)
    dirty = torch.zeros((96, 80), dtype=torch.complex128, device="cuda")
    plan.ms2dirty_chan(uvw, FREQS, to_dev(torch, vis), to_dev(torch, wgt), dirty)
    img = synth.random_image(96, 80, seed=8)
    vout = torch.zeros(vis.shape, dtype=torch.complex128, device="cuda")
    plan.dirty2ms_chan(uvw, FREQS, to_dev(torch, img), to_dev(torch, wgt), vout)
    torch.cuda.synchronize()
    plan.close()
    # <dirty2ms(img), vis> = <img, ms2dirty(vis)> (each side carries the weights once)
    lhs = np.vdot(vout.cpu().numpy(), vis).real
    rhs = np.vdot(img, dirty.cpu().numpy()).real
    assert abs(lhs - rhs) <= 1e-12 * abs(rhs)


def test_single_channel_identity(torch_cuda):
    torch = torch_cuda
    d, vis, wgt = _data(1, seed=9)
    outs = []
    for chan in (False, True):
        plan = Plan(96, 80, d["fov"], 1e-5, precision="fp32")
        uvw = to_dev(torch, d["uvw"], np.float64)
        v = to_dev(torch, vis, np.complex64)
        w = to_dev(torch, wgt, np.float32)
        dirty = torch.zeros((96, 80), dtype=torch.complex64, device="cuda")
        if chan:
            plan.ms2dirty_chan(uvw, [FREQS[0]], v, w, dirty)
        else:
            plan.ms2dirty(uvw, FREQS[0], v.reshape(-1), w.reshape(-1), dirty)
        torch.cuda.synchronize()
        outs.append(dirty.cpu().numpy())
        plan.close()
    assert np.array_equal(outs[0], outs[1])


def test_multichannel_rejects_bad_frequencies(torch_cuda):
    torch = torch_cuda
    d, vis, wgt = _data(2, nrow=100)
    plan = Plan(96, 80, d["fov"], 1e-5, precision="fp64")
    uvw = to_dev(torch, d["uvw"], np.float64)
    dirty = torch.zeros((96, 80), dtype=torch.complex128, device="cuda")
    with pytest.raises(GridderError):
        plan.ms2dirty_chan(uvw, [1e8, -1.0], to_dev(torch, vis), None, dirty)
    plan.close()
