"""Memory-limited mode (cg_plan_set_grid_budget): w planes processed window by
window (the reference's plane-cube loop, ra_exec.cu:292-389 and 522-613) give
the oracle's results and the resident path's, in both directions."""
import numpy as np
import pytest

from cugridder_b200 import GridderError, Plan, synth
from cugridder_b200.synth import rel_l2

from tests.gpu_helpers import to_dev

pytestmark = pytest.mark.gpu


def _run(torch, d, img, precision, budget, kernel=None):
    cdt = np.complex128 if precision == "fp64" else np.complex64
    rdt = np.float64 if precision == "fp64" else np.float32
    tc = torch.complex128 if precision == "fp64" else torch.complex64
    plan = Plan(d["nx"], d["ny"], d["fov"], 1e-5 if precision == "fp32" else 1e-9, precision=precision)
    if kernel is not None:
        plan.set_kernel("poly", kernel.W, kernel.horner)
    if budget:
        plan.set_grid_budget(budget)
    uvw = to_dev(torch, d["uvw"], np.float64)
    wgt = to_dev(torch, d["wgt"], rdt)
    dirty = torch.zeros((d["nx"], d["ny"]), dtype=tc, device="cuda")
    plan.ms2dirty(uvw, d["freq"], to_dev(torch, d["vis"], cdt), wgt, dirty)
    vis = torch.zeros(d["uvw"].shape[0], dtype=tc, device="cuda")
    plan.dirty2ms(uvw, d["freq"], to_dev(torch, img, cdt), wgt, vis)
    torch.cuda.synchronize()
    info = plan.info()
    plan.close()
    return dirty.cpu().numpy(), vis.cpu().numpy(), info


def _eps(precision):
    return 1e-5 if precision == "fp32" else 1e-9


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
@pytest.mark.parametrize("planes_per_window", [1, 3])
@pytest.mark.parametrize("case", ["c1_160x128", "wrap_122x250"])
def test_windows_match_oracle_and_resident(torch_cuda, oracle, precision, tol, planes_per_window,
                                           case):
    """Both directions against the oracle (FP64: 1e-10; FP32: 2e-5) and
    against the resident path; the second case has rows over the whole band
    and past it on a grid with partial last hives (nf 250 x 500)."""
    if case == "c1_160x128":
        d = synth.make("ms2dirty_256_fp64", seed=13, nrow=30000, nx=160, ny=128)
    else:
        d = synth.wrap_case(30000, 122, 250, 3.0, seed=19)
    nx, ny = d["nx"], d["ny"]
    img = synth.random_image(nx, ny, seed=14)
    ref = _run(torch_cuda, d, img, precision, 0)
    info = ref[2]
    tsz = 16 if precision == "fp64" else 8
    budget = planes_per_window * info["nf1"] * info["nf2"] * tsz
    got = _run(torch_cuda, d, img, precision, budget)
    assert got[2]["nw"] == info["nw"] and info["nw"] > planes_per_window
    assert rel_l2(got[0], ref[0]) < tol
    assert rel_l2(got[1], ref[1]) < tol
    eps = _eps(precision)
    ora_tol = 1e-10 if precision == "fp64" else 2e-5
    o_d, _ = oracle.ms2dirty(d["uvw"], d["vis"], d["wgt"], nx, ny, d["fov"], d["freq"], eps)
    o_v, _ = oracle.dirty2ms(d["uvw"], img, d["wgt"], d["fov"], d["freq"], eps)
    assert rel_l2(got[0], o_d) < ora_tol
    assert rel_l2(got[1], o_v) < ora_tol


def test_windows_with_learned_kernel(torch_cuda):
    from cugridder_b200.learn import available_widths, load_kernel

    if 6 not in available_widths():
        pytest.skip("no learned kernel")
    k = load_kernel(6)
    d = synth.make("ms2dirty_256_fp64", seed=15, nrow=30000, nx=128, ny=128)
    img = synth.random_image(128, 128, seed=16)
    ref = _run(torch_cuda, d, img, "fp32", 0, k)
    got = _run(torch_cuda, d, img, "fp32", 2 * ref[2]["nf1"] * ref[2]["nf2"] * 8, k)
    assert rel_l2(got[0], ref[0]) < 1e-5 and rel_l2(got[1], ref[1]) < 1e-5
    from oracle import oracle as O

    O.set_kernel("poly", k.W, k.horner)
    try:
        o_d, _ = O.ms2dirty(d["uvw"], d["vis"], d["wgt"], 128, 128, d["fov"], d["freq"], 1e-5)
        o_v, _ = O.dirty2ms(d["uvw"], img, d["wgt"], d["fov"], d["freq"], 1e-5)
    finally:
        O.set_kernel("es")
    assert rel_l2(got[0], o_d) < 2e-5 and rel_l2(got[1], o_v) < 2e-5


def test_budget_below_one_plane(torch_cuda):
    d = synth.make("ms2dirty_256_fp64", seed=17, nrow=1000, nx=64, ny=64)
    with pytest.raises(GridderError):
        _run(torch_cuda, d, synth.random_image(64, 64, seed=1), "fp64", 1024)
