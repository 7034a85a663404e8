"""The reference-compatible host entry points with ordinary (pageable)
numpy buffers, as the reference's Python binding passes them: inputs and
outputs above the 2 MB threshold go through the pinned staging buffers in
8 MB chunks.  The results must equal, bit for bit, those of the same calls
on pinned copies of the same arrays (which the DMA engine reads directly),
and match the oracle."""
import numpy as np
import pytest

import cugridder_b200 as cg
from cugridder_b200 import synth
from cugridder_b200.synth import rel_l2

pytestmark = pytest.mark.gpu


def _pinned(torch, a):
    t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
    t.numpy()[...] = a
    return t.numpy()


def _case():
    # uvw 400k x 3 float64 (9.6 MB: two chunks), visibilities 6.4 MB, weights
    # 3.2 MB, a 512 x 512 complex128 image (4 MB)
    d = synth.make("ms2dirty_256_fp64", seed=61, nrow=400_000, nx=512, ny=512, fov=2.0)
    img = synth.random_image(512, 512, seed=62)
    return d, img


def _both(torch, d, img, fp32):
    out = {}
    for kind in ("pageable", "pinned"):
        if fp32:
            uvw, vis = d["uvw"].astype(np.float32), d["vis"].astype(np.complex64)
            wgt, im = d["wgt"].astype(np.float32), img.astype(np.complex64)
            dirty, vout = np.zeros((512, 512), np.complex64), np.zeros(d["uvw"].shape[0], np.complex64)
        else:
            uvw, vis, wgt, im = d["uvw"], d["vis"].astype(np.complex128), d["wgt"], img
            dirty, vout = np.zeros((512, 512), np.complex128), np.zeros(d["uvw"].shape[0], np.complex128)
        if kind == "pinned":
            uvw, vis, wgt, im = (_pinned(torch, a) for a in (uvw, vis, wgt, im))
            dirty, vout = _pinned(torch, dirty), _pinned(torch, vout)
        n = uvw.shape[0]
        f1 = cg.ms2dirtyf_2 if fp32 else cg.ms2dirty_2
        f2 = cg.dirty2msf_2 if fp32 else cg.dirty2ms_2
        assert f1(n, 512, 512, d["fov"], d["freq"], uvw, vis, wgt, dirty, 1e-6, 2.0, -1) == 0
        assert f2(n, 512, 512, d["fov"], d["freq"], uvw, vout, wgt, im, 1e-6, 2.0, -1) == 0
        out[kind] = (np.array(dirty), np.array(vout))
    return out


@pytest.mark.parametrize("fp32", [False, True])
def test_pageable_equals_pinned(torch_cuda, fp32):
    d, img = _case()
    _both(torch_cuda, d, img, fp32)  # first calls: the cached plan's tuning
    out = _both(torch_cuda, d, img, fp32)
    np.testing.assert_array_equal(out["pageable"][0], out["pinned"][0])
    np.testing.assert_array_equal(out["pageable"][1], out["pinned"][1])


def test_pageable_vs_oracle(torch_cuda, oracle):
    d, img = _case()
    out = _both(torch_cuda, d, img, False)["pageable"]
    ref_d, _ = oracle.ms2dirty(d["uvw"], d["vis"], d["wgt"], 512, 512, d["fov"], d["freq"], 1e-6)
    ref_v, _ = oracle.dirty2ms(d["uvw"], img, d["wgt"], d["fov"], d["freq"], 1e-6)
    assert rel_l2(out[0], ref_d) < 1e-10
    assert rel_l2(out[1], ref_v) < 1e-10
