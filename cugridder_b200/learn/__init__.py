"""Learned gridding kernel: an MLP phi_theta trained against the FP64 direct
sum with this package's own CUDA forward/backward kernels, then fitted to
piecewise degree-7 Horner polynomials that the gridder evaluates
(``Plan.set_kernel("poly", W, coef)``).

    from cugridder_b200.learn import load_kernel
    k = load_kernel(5)            # committed artifact kernels/learned_W5.json
    plan.set_kernel("poly", k.W, k.horner)
"""
from .model import (H, NTHETA, LearnedKernel, available_widths, es_horner, horner_fit,  # noqa: F401
                    init_theta, kernel_path, load_kernel, phi_np, smallest_width)
