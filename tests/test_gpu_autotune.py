"""Plan autotuning (cg_plan_set_autotune): the tuned tiling comes from the
candidate list, the results agree with the default tiling to FP32 rounding,
and later calls reuse the tuned tiling (identical results)."""
import numpy as np
import pytest

from cugridder_b200 import Plan, synth
from cugridder_b200.synth import rel_l2

from tests.gpu_helpers import to_dev

pytestmark = pytest.mark.gpu


def _calls(torch, d, img, autotune, ncalls):
    p = Plan(d["nx"], d["ny"], d["fov"], 1e-5, precision="fp32")
    p.set_autotune(autotune)
    uvw = to_dev(torch, d["uvw"], np.float64)
    vis = to_dev(torch, d["vis"], np.complex64)
    wgt = to_dev(torch, d["wgt"], np.float32)
    dimg = to_dev(torch, img, np.complex64)
    outs = []
    for _ in range(ncalls):
        dirty = torch.zeros((d["nx"], d["ny"]), dtype=torch.complex64, device="cuda")
        vout = torch.zeros(d["uvw"].shape[0], dtype=torch.complex64, device="cuda")
        p.ms2dirty(uvw, d["freq"], vis, wgt, dirty)
        p.dirty2ms(uvw, d["freq"], dimg, wgt, vout)
        torch.cuda.synchronize()
        outs.append((dirty.cpu().numpy(), vout.cpu().numpy()))
    tiling = p.tiling()
    p.close()
    return outs, tiling


def test_autotuned_plan_matches_default(torch_cuda):
    d = synth.make("wstack_2048_10M", seed=3, nrow=300_000, nx=512, ny=512, fov=1.0)
    img = synth.random_image(512, 512, seed=4, dtype=np.complex64)
    tuned, tiling = _calls(torch_cuda, d, img, True, 3)
    ref, ref_tiling = _calls(torch_cuda, d, img, False, 1)
    grid_t, degrid_t, ms = tiling
    assert ms[0] > 0 and ms[1] > 0
    assert grid_t[0] in (16, 32) and grid_t[1] in (8, 16, 32)
    assert degrid_t[3] in (256, 512, -1, -2, -3, -4)  # threads per CTA, or a TMA-staged variant
    assert ref_tiling[2] == (0.0, 0.0)
    for dirty, vis in tuned:
        assert rel_l2(dirty, ref[0][0]) < 1e-5
        assert rel_l2(vis, ref[0][1]) < 1e-5
    # calls after the tuning one use the same tiling: deterministic results
    np.testing.assert_array_equal(tuned[1][0], tuned[2][0])
    np.testing.assert_array_equal(tuned[1][1], tuned[2][1])
