"""Shared helpers of the GPU tests: run the plan API on device buffers."""
import numpy as np

from cugridder_b200 import Plan, synth


def payload(d, p, sign=-1):
    """Gridded strengths c_j = vis * wgt * exp(i o_c w_eff) of the reference's
    prestage (ra_exec.cu:103-111; cuft.cu:46-66), for the oracle's spreading."""
    w_eff = (d["uvw"][:, 2] * (d["freq"] / synth.C_LIGHT * sign)) * (2 * np.pi)
    c = d["vis"].astype(np.complex128)
    if d.get("wgt") is not None:
        c = c * d["wgt"].astype(np.float64)
    return c * np.exp(1j * p.o_center * w_eff)


def to_dev(torch, a, dtype=None):
    if a is None:
        return None
    if dtype is not None:
        a = np.asarray(a).astype(dtype)
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def plan_ms2dirty(torch, d, precision, eps, sign=-1, stop=0, nx=None, ny=None, fov=None,
                  freq=None, use_wgt=True):
    nx = nx or d["nx"]
    ny = ny or d["ny"]
    fov = fov or d["fov"]
    freq = freq or d["freq"]
    cdt = np.complex128 if precision == "fp64" else np.complex64
    rdt = np.float64 if precision == "fp64" else np.float32
    plan = Plan(nx, ny, fov, eps, sign=sign, precision=precision)
    uvw = to_dev(torch, d["uvw"], np.float64)
    vis = to_dev(torch, d["vis"], cdt)
    wgt = to_dev(torch, d["wgt"], rdt) if (use_wgt and d.get("wgt") is not None) else None
    dirty = torch.zeros((nx, ny), dtype=torch.complex128 if precision == "fp64" else torch.complex64,
                        device="cuda")
    if stop:
        plan.set_stop_stage(stop)
    st = plan.ms2dirty(uvw, freq, vis, wgt, dirty)
    torch.cuda.synchronize()
    return plan, dirty.cpu().numpy(), st


def plan_dirty2ms(torch, d, img, precision, eps, sign=-1, stop=0, use_wgt=True):
    cdt = np.complex128 if precision == "fp64" else np.complex64
    rdt = np.float64 if precision == "fp64" else np.float32
    nx, ny = img.shape
    plan = Plan(nx, ny, d["fov"], eps, sign=sign, precision=precision)
    uvw = to_dev(torch, d["uvw"], np.float64)
    dirty = to_dev(torch, img, cdt)
    wgt = to_dev(torch, d["wgt"], rdt) if (use_wgt and d.get("wgt") is not None) else None
    vis = torch.zeros(d["uvw"].shape[0], dtype=torch.complex128 if precision == "fp64" else torch.complex64,
                      device="cuda")
    if stop:
        plan.set_stop_stage(stop)
    st = plan.dirty2ms(uvw, d["freq"], dirty, wgt, vis)
    torch.cuda.synchronize()
    return plan, vis.cpu().numpy(), st
