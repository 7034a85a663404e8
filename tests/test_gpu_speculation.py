"""dirty2ms through the host entry points starts its plane fill and FFT on the
last call's geometry when the row count and frequency repeat, before uvw is
in; the call's own range pass confirms the geometry or discards that work.
Both outcomes must give exactly the results of calls that never speculate
(CG_SPECULATE=0): the same uvw again (confirmed), and new uvw with the same
rows and frequency but other ranges (discarded), in FP64 and FP32."""
import numpy as np
import pytest

import cugridder_b200 as cg
from cugridder_b200 import synth

pytestmark = pytest.mark.gpu


def _call(d, img, fp32):
    n = d["uvw"].shape[0]
    if fp32:
        vis = np.zeros(n, np.complex64)
        assert cg.dirty2msf_2(n, 256, 256, d["fov"], d["freq"], d["uvw"].astype(np.float32), vis,
                              d["wgt"].astype(np.float32), img.astype(np.complex64), 1e-5, 2.0,
                              -1) == 0
    else:
        vis = np.zeros(n, np.complex128)
        assert cg.dirty2ms_2(n, 256, 256, d["fov"], d["freq"], d["uvw"], vis, d["wgt"], img, 1e-5,
                             2.0, -1) == 0
    return vis


@pytest.mark.parametrize("fp32", [False, True])
def test_speculated_geometry_confirmed_and_discarded(torch_cuda, monkeypatch, fp32):
    a = synth.make("ms2dirty_256_fp64", seed=71, nrow=150_000)
    b = synth.make("ms2dirty_256_fp64", seed=72, nrow=150_000)
    b["freq"] = a["freq"]
    b["uvw"] = b["uvw"] * 1.3  # other u, v, w ranges: another geometry
    img = synth.random_image(256, 256, seed=73)
    # reference results, no speculation
    monkeypatch.setenv("CG_SPECULATE", "0")
    ref_a = _call(a, img, fp32)
    ref_b = _call(b, img, fp32)
    monkeypatch.delenv("CG_SPECULATE")
    _call(a, img, fp32)  # the geometry of a
    got_a = _call(a, img, fp32)  # same rows, frequency, ranges: confirmed
    got_b = _call(b, img, fp32)  # same rows and frequency, other ranges: discarded
    got_a2 = _call(a, img, fp32)  # and back
    np.testing.assert_array_equal(got_a, ref_a)
    np.testing.assert_array_equal(got_b, ref_b)
    np.testing.assert_array_equal(got_a2, ref_a)
