"""Train the learned gridding kernel on the GPU.

    python -m cugridder_b200.learn.train --W 4 5 6 7 [--sets 4096 --nvis 10000 --n 512]

Each W trains its own network.  The training problem is the one the kernel
serves: random visibility sets that the method generates itself (M points
uniform on an nf x nf periodic grid, nf = 2N, complex N(0,1) strengths) are
spread with the separable kernel phi(x) phi(y), transformed by a 2-D FFT and
divided by the kernel's Fourier transform, computed by the same
Gauss-Legendre quadrature the gridder uses (p = int(2 + 1.5 W) positive
nodes, as the reference's fourier_series_appro, deconv.cu:80-93).  The loss
is the relative squared error against the FP64 direct sum on 64 x 64 random
modes per set, F(k1, k2) = sum_j c_j exp(2 pi i (k1 x_j + k2 y_j) / nf),
evaluated by this package's FP64 CUDA kernel.

The network's forward and backward passes, the spreading and its adjoint
and the direct sums are this package's CUDA kernels (libcugridder.so,
cg_learn_*); torch provides device memory, the FFT (cuFFT) and the
optimizer.  After training the kernel is fitted to piecewise degree-7 Horner
polynomials (the form the gridder evaluates) and written to
cugridder_b200/kernels/learned_W<W>.json (+ .theta.bin).
"""
import argparse
import json
import math
import os
import time

import numpy as np

from .. import _lib
from .model import (NTHETA, LearnedKernel, beta0_for, horner_eval, horner_fit, init_theta,
                    kernel_path, phi_np)


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("training needs a CUDA device")
    return torch


def _stream(torch):
    return torch.cuda.current_stream().cuda_stream


def make_autograd_fns(torch):
    """torch.autograd.Functions around the CUDA kernels: the kernel values
    phi_theta(d) (forward / backward in theta) and the 2-D spreading (forward /
    adjoint in the kernel values)."""
    lib = _lib.load()

    class Phi(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta, d, beta0, W):
            d = d.contiguous()
            phi = torch.empty_like(d)
            _lib.check(lib.cg_learn_phi_forward(theta.data_ptr(), float(beta0), int(W), d.numel(),
                                                d.data_ptr(), phi.data_ptr(), _stream(torch)))
            ctx.save_for_backward(theta, d)
            ctx.beta0, ctx.W = float(beta0), int(W)
            return phi

        @staticmethod
        def backward(ctx, g):
            theta, d = ctx.saved_tensors
            g = g.contiguous()
            dth = torch.zeros_like(theta)
            _lib.check(lib.cg_learn_phi_backward(theta.data_ptr(), ctx.beta0, ctx.W, d.numel(),
                                                 d.data_ptr(), g.data_ptr(), dth.data_ptr(),
                                                 _stream(torch)))
            return dth, None, None, None

    class Spread(torch.autograd.Function):
        @staticmethod
        def forward(ctx, phx, phy, c, gx0, gy0, nf, W):
            B, M = gx0.shape
            grid = torch.zeros((B, nf, nf, 2), dtype=torch.float32, device=c.device)
            phx, phy = phx.contiguous(), phy.contiguous()
            _lib.check(lib.cg_learn_spread2d(B, M, W, nf, c.data_ptr(), gx0.data_ptr(),
                                             gy0.data_ptr(), phx.data_ptr(), phy.data_ptr(),
                                             grid.data_ptr(), _stream(torch)))
            ctx.save_for_backward(phx, phy, c, gx0, gy0)
            ctx.nf, ctx.W = nf, W
            return grid

        @staticmethod
        def backward(ctx, g):
            phx, phy, c, gx0, gy0 = ctx.saved_tensors
            B, M = gx0.shape
            g = g.contiguous()
            dphx, dphy = torch.empty_like(phx), torch.empty_like(phy)
            _lib.check(lib.cg_learn_spread2d_adjoint(B, M, ctx.W, ctx.nf, c.data_ptr(),
                                                     gx0.data_ptr(), gy0.data_ptr(), phx.data_ptr(),
                                                     phy.data_ptr(), g.data_ptr(), dphx.data_ptr(),
                                                     dphy.data_ptr(), _stream(torch)))
            return dphx, dphy, None, None, None, None, None

    return Phi, Spread


def gl_nodes(W):
    """Positive half of 2p Gauss-Legendre nodes on [-W/2, W/2], p = int(2 + 1.5 W),
    with the weights of sum_n 2 (W/2) w_n phi(d_n) cos(.) = integral of phi cos."""
    p = int(2 + 1.5 * W)
    x, w = np.polynomial.legendre.leggauss(2 * p)
    x, w = x[p:], w[p:]
    alpha = W / 2.0
    return alpha * x, 2.0 * alpha * w


class Sets:
    """Method-generated training sets with their FP64 direct-sum targets."""

    def __init__(self, torch, nsets, nvis, n, K, seed, device):
        lib = _lib.load()
        self.nf = 2 * n
        g = torch.Generator(device=device)
        g.manual_seed(seed)
        self.X = torch.rand((nsets, nvis), generator=g, dtype=torch.float64, device=device) * self.nf
        self.Y = torch.rand((nsets, nvis), generator=g, dtype=torch.float64, device=device) * self.nf
        c = torch.randn((nsets, nvis, 2), generator=g, dtype=torch.float64, device=device)
        self.c64 = c.contiguous()
        self.c32 = c.float().contiguous()
        half = n // 2
        k1 = torch.randint(-half, half, (nsets, K), generator=g, device=device, dtype=torch.int32)
        k2 = torch.randint(-half, half, (nsets, K), generator=g, device=device, dtype=torch.int32)
        self.k1 = k1[:, :, None].expand(nsets, K, K).reshape(nsets, K * K).contiguous()
        self.k2 = k2[:, None, :].expand(nsets, K, K).reshape(nsets, K * K).contiguous()
        F = torch.empty((nsets, K * K, 2), dtype=torch.float64, device=device)
        chunk = 64
        for s0 in range(0, nsets, chunk):
            s1 = min(nsets, s0 + chunk)
            _lib.check(lib.cg_learn_dft2(s1 - s0, nvis, self.nf, self.X[s0:s1].data_ptr(),
                                         self.Y[s0:s1].data_ptr(), self.c64[s0:s1].data_ptr(),
                                         K * K, self.k1[s0:s1].data_ptr(), self.k2[s0:s1].data_ptr(),
                                         F[s0:s1].data_ptr(), _stream(torch)))
        self.F = torch.view_as_complex(F)
        self.nsets, self.nvis = nsets, nvis


class Problem:
    def __init__(self, torch, W):
        self.torch = torch
        self.W = W
        self.beta0 = beta0_for(W)
        self.Phi, self.Spread = make_autograd_fns(torch)
        dn, wn = gl_nodes(W)
        self.dn = torch.tensor(dn, dtype=torch.float32, device="cuda")
        self.wn = torch.tensor(wn, dtype=torch.float64, device="cuda")
        self.dn64 = torch.tensor(dn, dtype=torch.float64, device="cuda")

    def taps(self, X):
        torch = self.torch
        W = self.W
        g0 = torch.floor(X - W / 2.0) + 1.0
        l = torch.arange(W, dtype=torch.float64, device=X.device)
        d = (g0[..., None] + l - X[..., None]).float()
        return g0.to(torch.int32).contiguous(), d.contiguous()

    def phihat(self, phn, k, nf):
        # sum_n 2 alpha w_n phi(d_n) cos(2 pi k d_n / nf), FP64
        torch = self.torch
        arg = (2.0 * math.pi / nf) * k.double()[..., None] * self.dn64
        return (torch.cos(arg) * (self.wn * phn.double())).sum(-1)

    def rel_err(self, theta, sets, s0, s1, phi_taps=None):
        """Relative squared error per set of sets [s0, s1) (differentiable in theta)."""
        torch = self.torch
        W, nf = self.W, sets.nf
        X, Y = sets.X[s0:s1], sets.Y[s0:s1]
        gx0, dx = self.taps(X)
        gy0, dy = self.taps(Y)
        if phi_taps is None:
            phx = self.Phi.apply(theta, dx.reshape(-1), self.beta0, W).reshape(dx.shape)
            phy = self.Phi.apply(theta, dy.reshape(-1), self.beta0, W).reshape(dy.shape)
            phn = self.Phi.apply(theta, self.dn, self.beta0, W)
        else:
            phx, phy, phn = phi_taps(dx), phi_taps(dy), phi_taps(self.dn)
        u = self.Spread.apply(phx, phy, sets.c32[s0:s1], gx0, gy0, nf, W)
        U = torch.fft.ifft2(torch.view_as_complex(u), dim=(1, 2)) * float(nf * nf)
        k1, k2 = sets.k1[s0:s1].long(), sets.k2[s0:s1].long()
        b = torch.arange(s1 - s0, device=U.device)[:, None]
        Uk = U[b, k1 % nf, k2 % nf].to(torch.complex128)
        fk = Uk / (self.phihat(phn, k1, nf) * self.phihat(phn, k2, nf))
        F = sets.F[s0:s1]
        return ((fk - F).abs() ** 2).sum(1) / (F.abs() ** 2).sum(1)


def train_one(torch, W, nsets=4096, nvis=10000, n=512, K=64, batch=16, epochs=16, lr=3e-3,
              seed=0, log=print):
    t0 = time.time()
    sets = Sets(torch, nsets, nvis, n, K, seed=1000 + W, device="cuda")
    test = Sets(torch, 64, nvis, n, K, seed=5000 + W, device="cuda")
    torch.cuda.synchronize()
    t_data = time.time() - t0
    prob = Problem(torch, W)
    theta = torch.tensor(init_theta(seed + W), dtype=torch.float32, device="cuda", requires_grad=True)
    zero = torch.zeros(NTHETA, dtype=torch.float32, device="cuda")

    def evaluate(th):
        with torch.no_grad():
            e = torch.cat([prob.rel_err(th, test, s, min(s + batch, test.nsets))
                           for s in range(0, test.nsets, batch)])
        return float(e.mean().sqrt())

    err_es = evaluate(zero)
    opt = torch.optim.Adam([theta], lr=lr)
    steps = epochs * (nsets // batch)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, steps, eta_min=lr * 0.02)
    hist = []
    step = 0
    best = (err_es, zero.clone())
    for ep in range(epochs):
        order = torch.randperm(nsets // batch).tolist()
        for bi in order:
            s0 = bi * batch
            loss = torch.log(prob.rel_err(theta, sets, s0, s0 + batch).mean())
            opt.zero_grad(set_to_none=True)
            loss.backward()
            opt.step()
            sched.step()
            step += 1
        e = evaluate(theta.detach())
        hist.append({"epoch": ep + 1, "step": step, "test_rel_l2": e})
        log("W=%d epoch %d: test rel L2 %.3e (ES %.3e)" % (W, ep + 1, e, err_es))
        if e < best[0]:
            best = (e, theta.detach().clone())
    th = best[1].double().cpu().numpy()
    coef = horner_fit(lambda d: phi_np(th, prob.beta0, W, d), W)
    dn = np.linspace(-W / 2 + 1e-9, W / 2 - 1e-9, 20001)
    ref = phi_np(th, prob.beta0, W, dn)
    fit_err = float(np.abs(horner_eval(coef, W, dn) - ref).max() / np.abs(ref).max())

    def horner_taps(d):
        v = horner_eval(coef, W, d.double().cpu().numpy())
        return torch.tensor(v, dtype=torch.float32, device="cuda")

    with torch.no_grad():
        e_h = torch.cat([prob.rel_err(None, test, s, min(s + batch, test.nsets), phi_taps=horner_taps)
                         for s in range(0, test.nsets, batch)])
    err_horner = float(e_h.mean().sqrt())
    meta = {
        "train": {"sets": nsets, "vis_per_set": nvis, "image": [n, n], "grid": [2 * n, 2 * n],
                  "modes_per_set": K * K, "batch": batch, "epochs": epochs, "steps": step, "lr": lr,
                  "seed": seed, "optimizer": "Adam + cosine decay",
                  "loss": "log mean relative squared error vs FP64 direct sum",
                  "seconds": round(time.time() - t0, 1), "seconds_data": round(t_data, 1)},
        "eval_2d": {"test_sets": test.nsets, "rel_l2_es": err_es, "rel_l2_learned": best[0],
                    "rel_l2_learned_horner": err_horner, "horner_max_rel_fit_error": fit_err,
                    "gain_over_es": err_es / best[0] if best[0] > 0 else None},
        "history": hist,
    }
    return LearnedKernel(W, prob.beta0, th, coef, meta)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--W", type=int, nargs="+", default=[4, 5, 6, 7, 8])
    ap.add_argument("--sets", type=int, default=4096)
    ap.add_argument("--nvis", type=int, default=10000)
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--epochs", type=int, default=16)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--out", default=None, help="directory (default: the package's kernels/)")
    a = ap.parse_args()
    torch = _torch()
    for W in a.W:
        k = train_one(torch, W, nsets=a.sets, nvis=a.nvis, n=a.n, batch=a.batch, epochs=a.epochs,
                      lr=a.lr)
        path = kernel_path(W, a.out)
        os.makedirs(os.path.dirname(path), exist_ok=True)
        k.save(path)
        print(json.dumps({"W": W, **k.meta["eval_2d"], "seconds": k.meta["train"]["seconds"]}),
              flush=True)


if __name__ == "__main__":
    main()
