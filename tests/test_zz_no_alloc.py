"""cg_bin_static (allocation-free hive binning) against the plan path.

The plan path (cg_plan_ms2dirty stopped after binning, buffers read back
with cg_plan_copy_buffer) is the existing entry point; cg_bin_static must
produce the same permutation and hive offsets bit for bit, on two calls in a
row with different inputs (so no state of the first call leaks into the
second).  Kept in the last-collected file so it also runs after every other
GPU test in one process.
"""
import ctypes

import numpy as np
import pytest

from cugridder_b200 import Plan, _lib, synth

pytestmark = pytest.mark.gpu

CG_ERR_SIZE = 6


def _plan_binning(torch, d, precision, eps, sign, grid_budget=0):
    cdt = np.complex128 if precision == "fp64" else np.complex64
    rdt = np.float64 if precision == "fp64" else np.float32
    plan = Plan(d["nx"], d["ny"], d["fov"], eps, sign=sign, precision=precision)
    try:
        if grid_budget:
            plan.set_grid_budget(grid_budget)
        uvw = torch.from_numpy(d["uvw"]).cuda()
        vis = torch.from_numpy(d["vis"].astype(cdt)).cuda()
        wgt = torch.from_numpy(d["wgt"].astype(rdt)).cuda()
        dirty = torch.zeros((d["nx"], d["ny"]), dtype=torch.complex128 if precision == "fp64"
                            else torch.complex64, device="cuda")
        plan.set_stop_stage(1)
        plan.ms2dirty(uvw, d["freq"], vis, wgt, dirty)
        torch.cuda.synchronize()
        return plan.copy_buffer(_lib.CG_BUF_PERM), plan.copy_buffer(_lib.CG_BUF_HIVE_START)
    finally:
        plan.close()


def _static_binning(torch, lib, d, precision, eps, sign):
    prec = _lib.CG_PREC_FP64 if precision == "fp64" else _lib.CG_PREC_FP32
    nrow = d["uvw"].shape[0]
    uvw = torch.from_numpy(d["uvw"]).cuda()
    perm = torch.full((nrow,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    nh = ctypes.c_int64(0)
    args = (nrow, d["nx"], d["ny"], float(d["fov"]), float(d["freq"]), uvw.data_ptr(), eps, 2.0,
            sign, prec, perm.data_ptr())
    # size query: no hive_start buffer -> CG_ERR_SIZE with n_hives stored
    r = lib.cg_bin_static(*args, None, 0, ctypes.byref(nh), stream)
    assert r == CG_ERR_SIZE and nh.value > 0
    hs = torch.full((nh.value + 1,), -1, dtype=torch.int32, device="cuda")
    r = lib.cg_bin_static(*args, hs.data_ptr(), nh.value + 1, ctypes.byref(nh), stream)
    _lib.check(r)
    torch.cuda.synchronize()
    return perm.cpu().numpy(), hs.cpu().numpy()


@pytest.mark.parametrize("precision,eps,sign", [("fp32", 1e-5, -1), ("fp64", 1e-9, 1)])
def test_static_binning_matches_plan_two_calls(torch_cuda, precision, eps, sign):
    torch = torch_cuda
    lib = _lib.load()
    cap = lib.cg_bin_static_max_rows()
    assert cap == 524288
    first = synth.make("wstack_2048_10M", seed=11, nrow=cap, nx=1024, ny=1024, fov=2.0)
    second = synth.make("wstack_2048_10M", seed=12, nrow=150_001, nx=768, ny=640, fov=3.0,
                        w_max=300.0)
    for d in (first, second):
        p_ref, h_ref = _plan_binning(torch, d, precision, eps, sign)
        p, h = _static_binning(torch, lib, d, precision, eps, sign)
        assert p.shape == p_ref.shape and h.shape == h_ref.shape
        np.testing.assert_array_equal(p, p_ref)
        np.testing.assert_array_equal(h, h_ref)
        assert h[-1] == d["uvw"].shape[0]
        assert np.array_equal(np.sort(p), np.arange(d["uvw"].shape[0], dtype=np.int32))


def test_static_binning_eight_byte_keys_at_cap(torch_cuda, oracle):
    """nhx * nhy * nw * 64 > 2^32 (4096^2 image, w up to 20 km: 84 planes of
    1024^2 hives), so both paths sort 64-bit cell keys; at the row cap that
    layout fills most of the 15 MiB array.  Bit for bit against the plan path
    (whose grid is held to a 2 GiB budget of planes: binning only)."""
    torch = torch_cuda
    lib = _lib.load()
    cap = lib.cg_bin_static_max_rows()
    d = synth.make("wstack_4096_20M", seed=13, nrow=cap, w_max=20000.0)
    p = oracle.setup(d["uvw"], d["nx"], d["ny"], d["fov"], d["freq"], 1e-5, eps_floor=6e-8)
    nh = p.nhive[0] * p.nhive[1] * p.nhive[2]
    assert nh * 64 > 2 ** 32
    keys = oracle.bin_keys(p, d["uvw"])
    assert keys.max() >= 2 ** 32  # rows whose keys need the upper word
    p_ref, h_ref = _plan_binning(torch, d, "fp32", 1e-5, -1, grid_budget=2 << 30)
    for _ in range(2):
        perm, hs = _static_binning(torch, lib, d, "fp32", 1e-5, -1)
        np.testing.assert_array_equal(perm, p_ref)
        np.testing.assert_array_equal(hs, h_ref)
    assert hs.size == nh + 1 and hs[-1] == cap
    np.testing.assert_array_equal(perm, np.argsort(keys, kind="stable"))


def test_static_binning_rejects_oversize(torch_cuda):
    torch = torch_cuda
    lib = _lib.load()
    cap = lib.cg_bin_static_max_rows()
    perm = torch.full((4,), -7, dtype=torch.int32, device="cuda")
    hs = torch.full((4,), -7, dtype=torch.int32, device="cuda")
    nh = ctypes.c_int64(-1)
    # the row-count check runs before any pointer is read
    r = lib.cg_bin_static(cap + 1, 1024, 1024, 2.0, 1.5e8, perm.data_ptr(), 1e-5, 2.0, -1,
                          _lib.CG_PREC_FP32, perm.data_ptr(), hs.data_ptr(), 4, ctypes.byref(nh),
                          None)
    assert r == CG_ERR_SIZE
    assert b"524288" in lib.cg_last_error()
    torch.cuda.synchronize()
    assert (perm.cpu().numpy() == -7).all() and (hs.cpu().numpy() == -7).all()
