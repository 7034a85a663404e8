"""Host entry points (cg_ms2dirty_mixed / cg_dirty2ms_mixed) with the
learned kernel selected by cg_set_host_kernel, against a device plan with
the same kernel; and back to ES afterwards."""
import numpy as np
import pytest

from cugridder_b200 import Plan, dirty2ms_mixed, ms2dirty_mixed, set_host_kernel, synth
from cugridder_b200.synth import rel_l2

from tests.gpu_helpers import to_dev

pytestmark = pytest.mark.gpu


def test_host_api_learned_kernel_matches_plan(torch_cuda):
    from cugridder_b200.learn import load_kernel

    torch = torch_cuda
    k = load_kernel(6)
    d = synth.make("wstack_2048_10M", seed=21, nrow=200_000, nx=512, ny=512, fov=1.0)
    vis = d["vis"].astype(np.complex64)
    wgt = d["wgt"].astype(np.float32)
    img = synth.random_image(512, 512, seed=22, dtype=np.complex64)
    set_host_kernel("poly", k.W, k.horner)
    try:
        dirty_h = ms2dirty_mixed(d["uvw"], d["freq"], vis, wgt, 512, 512, 1.0, 1e-5)
        vis_h = dirty2ms_mixed(d["uvw"], d["freq"], img, wgt, 1.0, 1e-5)
    finally:
        set_host_kernel("es")
    p = Plan(512, 512, 1.0, 1e-5, precision="fp32")
    p.set_kernel("poly", k.W, k.horner)
    uvw = to_dev(torch, d["uvw"], np.float64)
    dirty = torch.zeros((512, 512), dtype=torch.complex64, device="cuda")
    p.ms2dirty(uvw, d["freq"], to_dev(torch, vis), to_dev(torch, wgt), dirty)
    vout = torch.zeros(d["uvw"].shape[0], dtype=torch.complex64, device="cuda")
    p.dirty2ms(uvw, d["freq"], to_dev(torch, img), to_dev(torch, wgt), vout)
    torch.cuda.synchronize()
    assert p.info()["kw"] == 6
    p.close()
    assert rel_l2(dirty_h, dirty.cpu().numpy()) < 1e-6
    assert rel_l2(vis_h, vout.cpu().numpy()) < 1e-6
    # back to ES: the host call now differs from the learned-kernel result
    dirty_es = ms2dirty_mixed(d["uvw"], d["freq"], vis, wgt, 512, 512, 1.0, 1e-5)
    assert rel_l2(dirty_es, dirty_h) > 1e-7
