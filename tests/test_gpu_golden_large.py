"""Full-size parity against the REFERENCE's own outputs and the FP64 DFT.

tests/golden/ref_large.npz holds what the reference's own CUDA build
(oracle/_ref/libcurafft_ref.so through its ms2dirty_2 / dirty2ms_2 and
ms2dirtyf_2 / dirty2msf_2, src/astro/cugridder.cu:541-571) returned on the
4096^2 / 20M-row workload (fov 5 deg, 1.5e8 Hz) and on the 2048^2 / 10M-row
workload (fov 3 deg), kept on a seeded subset of 4096 pixels and 4096 rows
(tests/golden/make_golden.py --large-out).  The inputs are regenerated here from
their seeds and checked against the recorded checksums.

Bars (relative L2 on the subsets):
- within 2 eps of the reference's FP64 output at the same eps;
- within 2 eps of the FP64 direct sums (cg_explicit_*, which must match the
  oracle's CPU sums recorded with the golden to 1e-12), or, where the
  reference's own output is itself farther than eps from them (the ES
  kernel's error at W = 10 for eps 1e-9), within the reference's own error
  plus eps;
- the reference's FP32 build, whose coordinates are FP32 too: within 2 eps
  plus its own distance from its FP64 output;
- the adjoint identity <dirty2ms(d), v> = <d, ms2dirty(v)> to 1e-6 relative
  in FP32.

tests/golden/ref_bins.npz holds the reference's binning (bin_mapping, via
oracle/ref_bins.cu): the hive offsets and the rows per grid cell, which this
library's binning must reproduce bit for bit.
"""
import hashlib
import os

import numpy as np
import pytest

from cugridder_b200 import Plan, _lib, synth
from cugridder_b200.synth import rel_l2

from tests.golden.make_golden import bin_cases, canon_cells, sha

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
LARGE = os.path.join(HERE, "golden", "ref_large.npz")
BINS = os.path.join(HERE, "golden", "ref_bins.npz")


def _load(path):
    if not os.path.exists(path):
        pytest.skip("golden record %s not present" % os.path.basename(path))
    return dict(np.load(path))


@pytest.fixture(scope="module")
def large():
    return _load(LARGE)


@pytest.fixture(scope="module")
def bins():
    return _load(BINS)


def _explicit(torch, d, img, pix, rows):
    """FP64 direct sums on the device for the pixel and row subsets."""
    lib = _lib.load()
    dev = torch.device("cuda")
    M = d["uvw"].shape[0]
    st = torch.cuda.current_stream().cuda_stream
    uvw = torch.from_numpy(d["uvw"]).to(dev)
    vis = torch.from_numpy(d["vis"].astype(np.complex128)).to(dev)
    wgt = torch.from_numpy(d["wgt"].astype(np.float64)).to(dev)
    dimg = torch.from_numpy(img.astype(np.complex128)).to(dev)
    tp, tr = torch.from_numpy(pix).to(dev), torch.from_numpy(rows).to(dev)
    rd = torch.empty(pix.size, dtype=torch.complex128, device=dev)
    rv = torch.empty(rows.size, dtype=torch.complex128, device=dev)
    _lib.check(lib.cg_explicit_ms2dirty(M, d["nx"], d["ny"], d["fov"], d["freq"], uvw.data_ptr(),
                                        vis.data_ptr(), wgt.data_ptr(), -1, pix.size, tp.data_ptr(),
                                        rd.data_ptr(), st))
    _lib.check(lib.cg_explicit_dirty2ms(M, d["nx"], d["ny"], d["fov"], d["freq"], uvw.data_ptr(),
                                        dimg.data_ptr(), wgt.data_ptr(), -1, rows.size,
                                        tr.data_ptr(), rv.data_ptr(), st))
    torch.cuda.synchronize()
    return rd.cpu().numpy(), rv.cpu().numpy()


def _run(torch, d, img, precision, eps, kernel=None):
    """ms2dirty + dirty2ms through the plan API on device buffers; returns
    the full image and visibilities (complex128 on the host)."""
    cdt = torch.complex128 if precision == "fp64" else torch.complex64
    rdt = torch.float64 if precision == "fp64" else torch.float32
    nx, ny = d["nx"], d["ny"]
    with Plan(nx, ny, d["fov"], eps, precision=precision) as p:
        if kernel is not None:
            p.set_kernel("poly", kernel.W, kernel.horner)
        uvw = torch.from_numpy(d["uvw"]).cuda()
        vis = torch.from_numpy(d["vis"]).to(device="cuda", dtype=cdt)
        wgt = torch.from_numpy(d["wgt"]).to(device="cuda", dtype=rdt)
        dirty = torch.zeros((nx, ny), dtype=cdt, device="cuda")
        p.ms2dirty(uvw, d["freq"], vis, wgt, dirty)
        out = torch.zeros(d["uvw"].shape[0], dtype=cdt, device="cuda")
        p.dirty2ms(uvw, d["freq"], torch.from_numpy(img).to(device="cuda", dtype=cdt), wgt, out)
        torch.cuda.synchronize()
        W = p.info()["kw"]
        res = dirty.cpu().numpy().astype(np.complex128), out.cpu().numpy().astype(np.complex128)
    del uvw, vis, wgt, dirty, out
    torch.cuda.empty_cache()
    return res, W


CASES = {"c2": ("wstack_4096_20M", 20_000_000), "c4": ("wstack_2048_10M", 10_000_000)}


@pytest.fixture(scope="module")
def workloads(large):
    out = {}
    for name, (cfg, nrow) in CASES.items():
        d = synth.make(cfg, seed=0, nrow=nrow)
        img = synth.random_image(d["nx"], d["ny"], seed=1000, dtype=np.complex64)
        assert sha(d["uvw"], d["vis"], d["wgt"], img) == str(large[name + "/sha_inputs"]), name
        out[name] = (d, img)
    return out


# (case, our precision, eps, our kernel, reference record at the same eps)
FORMS = [("c2", "fp32", 1e-5, "learned", "fp64_1e-05"),
         ("c2", "fp32", 1e-5, "es", "fp64_1e-05"),
         ("c2", "fp64", 1e-9, "es", "fp64_1e-09"),
         ("c4", "fp32", 1e-5, "learned", "fp64_1e-05"),
         ("c4", "fp32", 1e-4, "learned", "fp64_0.0001"),
         ("c4", "fp64", 1e-4, "es", "fp64_0.0001")]


@pytest.mark.parametrize("case,precision,eps,kernel,refkey", FORMS)
def test_full_size_vs_reference_and_dft(torch_cuda, large, workloads, case, precision, eps,
                                        kernel, refkey):
    d, img = workloads[case]
    pix, rows = large[case + "/pixels"], large[case + "/rows"]
    assert (large["%s/%s/status" % (case, refkey)] == 0).all()
    k = None
    if kernel == "learned":
        from cugridder_b200.learn import smallest_width

        k = smallest_width(eps)
    (dirty, vis), _ = _run(torch_cuda, d, img, precision, eps, kernel=k)
    ds, vs = dirty.reshape(-1)[pix], vis[rows]
    ref_d, ref_v = large["%s/%s/dirty" % (case, refkey)], large["%s/%s/vis" % (case, refkey)]
    dft_d, dft_v = _explicit(torch_cuda, d, img, pix, rows)
    if case + "/dft_dirty" in large:
        # the oracle's CPU direct sums recorded with the golden: the on-device
        # sums must agree with them to FP64 rounding at full size
        assert rel_l2(dft_d, large[case + "/dft_dirty"]) < 1e-12
        assert rel_l2(dft_v, large[case + "/dft_vis"]) < 1e-12
    tol = 2 * eps
    assert rel_l2(ds, ref_d) < tol and rel_l2(vs, ref_v) < tol, (rel_l2(ds, ref_d), rel_l2(vs, ref_v))
    # against the DFT: 2 eps, or, where the reference's own output at this eps
    # is itself farther than eps from the DFT (the ES kernel's error at its
    # width), no more than eps beyond the reference's own error
    ref_err = max(rel_l2(ref_d, dft_d), rel_l2(ref_v, dft_v))
    tol_dft = max(tol, ref_err + eps)
    assert rel_l2(ds, dft_d) < tol_dft and rel_l2(vs, dft_v) < tol_dft, (
        rel_l2(ds, dft_d), rel_l2(vs, dft_v), ref_err)
    if precision == "fp32" and eps == 1e-5:
        # the reference's FP32 build (FP32 coordinates): 2 eps plus its own
        # distance from its FP64 output at the same eps
        r32d, r32v = large["%s/fp32_1e-05/dirty" % case], large["%s/fp32_1e-05/vis" % case]
        assert (large["%s/fp32_1e-05/status" % case] == 0).all()
        assert rel_l2(ds, r32d) < tol + rel_l2(r32d, ref_d)
        assert rel_l2(vs, r32v) < tol + rel_l2(r32v, ref_v)


def test_full_size_adjointness_fp32(torch_cuda, workloads):
    """<dirty2ms(d), v> = <d, ms2dirty(v)> on the 4096^2 / 20M workload, learned
    FP32 form, to 1e-6 relative."""
    from cugridder_b200.learn import smallest_width

    d, img = workloads["c2"]
    (dirty, vis), _ = _run(torch_cuda, d, img, "fp32", 1e-5, kernel=smallest_width(1e-5))
    lhs = np.vdot(vis, d["vis"].astype(np.complex128))
    rhs = np.vdot(img.astype(np.complex128), dirty)
    assert abs(lhs - rhs) <= 1e-6 * abs(rhs)


@pytest.mark.parametrize("name", [c[0] for c in bin_cases()])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_binning_vs_reference_bin_mapping(torch_cuda, bins, name, precision):
    """Hive offsets (the reference's plan->hive_count) and the rows per cell
    (the reference's histogram) bit for bit: our CG_BUF_HIVE_START and the
    run lengths of our sorted keys.  The FP32 plan bins from the same FP64
    coordinates, so it must agree too."""
    c = dict(bin_cases())[name]
    assert sha(c["uvw"]) == str(bins[name + "/sha_uvw"])
    assert bins[name + "/status"].item() == 0 and bins[name + "/method"].item() in (2, 6)
    nrow = c["uvw"].shape[0]
    cdt = torch_cuda.complex128 if precision == "fp64" else torch_cuda.complex64
    with Plan(c["nx"], c["ny"], c["fov"], c["eps"], precision=precision) as p:
        uvw = torch_cuda.from_numpy(c["uvw"]).cuda()
        vis = torch_cuda.zeros(nrow, dtype=cdt, device="cuda")
        dirty = torch_cuda.zeros((c["nx"], c["ny"]), dtype=cdt, device="cuda")
        p.set_stop_stage(1)
        p.ms2dirty(uvw, c["freq"], vis, None, dirty)
        torch_cuda.cuda.synchronize()
        inf = p.info()
        hs = p.copy_buffer(_lib.CG_BUF_HIVE_START).astype(np.int32)
        keys = p.copy_buffer(_lib.CG_BUF_SORTED_KEYS).astype(np.uint64)
    assert [inf["nf1"], inf["nf2"], inf["nw"]] == bins[name + "/nf"].tolist()
    assert list(inf["nhive"]) == bins[name + "/nhive"].tolist()
    if name + "/hive_count" in bins:
        np.testing.assert_array_equal(hs, bins[name + "/hive_count"])
    assert hashlib.sha256(hs.astype("<i4").tobytes()).hexdigest() == str(bins[name + "/hive_sha"])
    assert np.all(keys[1:] >= keys[:-1])
    uk, cnt = np.unique(keys, return_counts=True)
    assert uk.size == bins[name + "/ncells"].item()
    assert canon_cells(uk, cnt) == str(bins[name + "/cells_sha"])
