"""Generic NUFFT (type 1 / 2, 1-3 dimensions) against direct sums, with the
conventions of the reference's test/nufft_*_test.cu (modes k - N/2, k1
fastest, coordinates in radians)."""
import numpy as np
import pytest

from cugridder_b200.nufft import NufftPlan
from cugridder_b200.synth import rel_l2

from tests.gpu_helpers import to_dev

pytestmark = pytest.mark.gpu


def _phase(coords, nmodes, iflag):
    """exp(i iflag sum_d (k_d - N_d/2) x_d) as [M, prod N] with k1 fastest."""
    grids = np.meshgrid(*[np.arange(n) - n // 2 for n in reversed(nmodes)], indexing="ij")
    ks = [g.reshape(-1) for g in reversed(grids)]  # k1 varies fastest
    arg = sum(np.outer(x, k) for x, k in zip(coords, ks))
    return np.exp(1j * iflag * arg)


CASES = [((64,), 3000), ((48, 40), 2000), ((16, 12, 10), 1500)]


@pytest.mark.parametrize("precision,eps,tol", [("fp64", 1e-9, 5e-9), ("fp32", 1e-5, 5e-5)])
@pytest.mark.parametrize("nmodes,M", CASES)
@pytest.mark.parametrize("ntype,iflag", [(1, 1), (2, -1)])
def test_nufft_vs_direct(torch_cuda, precision, eps, tol, nmodes, M, ntype, iflag):
    torch = torch_cuda
    rng = np.random.Generator(np.random.PCG64(len(nmodes) * 10 + ntype))
    coords = [rng.uniform(-np.pi, np.pi, M) for _ in nmodes]
    E = _phase(coords, nmodes, iflag)
    cdt = np.complex128 if precision == "fp64" else np.complex64
    tc = torch.complex128 if precision == "fp64" else torch.complex64
    p = NufftPlan(ntype, nmodes, iflag=iflag, eps=eps, precision=precision)
    dc = [to_dev(torch, x) for x in coords]
    p.setpts(*dc)
    nk = int(np.prod(nmodes))
    if ntype == 1:
        c = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(cdt)
        fk = torch.zeros(nk, dtype=tc, device="cuda")
        p.execute(to_dev(torch, c), fk)
        ref = c.astype(np.complex128) @ E
        got = fk.cpu().numpy()
    else:
        f = (rng.standard_normal(nk) + 1j * rng.standard_normal(nk)).astype(cdt)
        cout = torch.zeros(M, dtype=tc, device="cuda")
        p.execute(cout, to_dev(torch, f))
        ref = E @ f.astype(np.complex128)
        got = cout.cpu().numpy()
    torch.cuda.synchronize()
    p.close()
    assert rel_l2(got, ref) < tol


@pytest.mark.parametrize("nmodes", [(50,), (32, 24), (12, 10, 8)])
def test_nufft_types_are_adjoint(torch_cuda, nmodes):
    torch = torch_cuda
    rng = np.random.Generator(np.random.PCG64(5))
    M = 1000
    coords = [to_dev(torch, rng.uniform(-np.pi, np.pi, M)) for _ in nmodes]
    nk = int(np.prod(nmodes))
    c = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    f = rng.standard_normal(nk) + 1j * rng.standard_normal(nk)
    p1 = NufftPlan(1, nmodes, iflag=1, eps=1e-12)
    p2 = NufftPlan(2, nmodes, iflag=-1, eps=1e-12)
    p1.setpts(*coords)
    p2.setpts(*coords)
    fk = torch.zeros(nk, dtype=torch.complex128, device="cuda")
    p1.execute(to_dev(torch, c), fk)
    cout = torch.zeros(M, dtype=torch.complex128, device="cuda")
    p2.execute(cout, to_dev(torch, f))
    torch.cuda.synchronize()
    lhs = np.vdot(f, fk.cpu().numpy())
    rhs = np.vdot(cout.cpu().numpy(), c)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    p1.close()
    p2.close()
