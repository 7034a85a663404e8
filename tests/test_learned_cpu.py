"""Learned kernel on the CPU: the oracle's FP64 MLP gradient against finite
differences, the numpy model against the oracle, the Horner fit, and the
oracle's piecewise-polynomial kernel path against its ES path."""
import numpy as np
import pytest

from cugridder_b200.learn import model as M


def _rand_theta(seed):
    th = M.init_theta(seed)
    rng = np.random.Generator(np.random.PCG64(seed + 100))
    o = 2 * M.H + M.H * M.H + M.H
    th[o:o + M.H] = rng.normal(0, 0.3, M.H)  # non-zero output layer
    th[-1] = 0.1
    return th


def test_oracle_mlp_matches_numpy(oracle):
    th = _rand_theta(1)
    d = np.linspace(-2.6, 2.6, 257)
    np.testing.assert_allclose(oracle.learn_phi(th, 13.8, 6, d), M.phi_np(th, 13.8, 6, d),
                               rtol=1e-13, atol=0)
    assert oracle.learn_phi(th, 13.8, 6, np.array([3.0, -3.2]))[0] == 0.0


def test_oracle_mlp_gradient_finite_differences(oracle):
    th = _rand_theta(2)
    rng = np.random.Generator(np.random.PCG64(3))
    W, beta0 = 5, 11.5
    d = rng.uniform(-2.5, 2.5, 200)
    g = rng.normal(size=200)
    grad = oracle.learn_phi_grad(th, beta0, W, d, g)

    def L(t):
        return float(np.dot(g, oracle.learn_phi(t, beta0, W, d)))

    idx = rng.choice(M.NTHETA, 40, replace=False)
    idx = np.concatenate([idx, [0, 32, 64, 64 + 1023, M.NTHETA - 1]])
    for i in idx:
        h = 1e-6
        tp, tm = th.copy(), th.copy()
        tp[i] += h
        tm[i] -= h
        fd = (L(tp) - L(tm)) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, grad[i])


# degree-7 fit error of ES (max 1), limited by the sqrt edge of the outer
# segments; each bound sits 20x or more below ES's own accuracy at that W
@pytest.mark.parametrize("W,tol", [(4, 5e-5), (5, 5e-6), (6, 1e-6), (7, 3e-7), (8, 1e-7)])
def test_horner_fit_of_es(W, tol):
    coef = M.es_horner(W)
    d = np.linspace(-W / 2 + 1e-9, W / 2 - 1e-9, 4001)
    ref = M.phi_np(np.zeros(M.NTHETA), M.beta0_for(W), W, d)
    assert np.abs(M.horner_eval(coef, W, d) - ref).max() < tol


def test_oracle_poly_kernel_matches_es(oracle):
    """The oracle's piecewise-polynomial path with the ES Horner table gives
    the ES result up to the fit error (ms2dirty, c1-like case)."""
    from cugridder_b200 import synth

    d = synth.make("ms2dirty_256_fp64", seed=4, nrow=3000)
    args = (d["uvw"], d["vis"], d["wgt"], 64, 64, d["fov"], d["freq"], 1e-5)
    ref, p_es = oracle.ms2dirty(*args)
    W = p_es.kw
    coef = M.horner_fit(lambda x: np.exp(p_es.beta * (np.sqrt(np.clip(1 - (2 * x / W) ** 2, 0, None)) - 1))
                        * (np.abs(x) < W / 2), W)
    oracle.set_kernel("poly", W, coef)
    try:
        got, p_poly = oracle.ms2dirty(*args)
    finally:
        oracle.set_kernel("es")
    assert p_poly.kern == 1 and p_poly.kw == W
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-5


def test_artifacts_load():
    from cugridder_b200.learn import available_widths, load_kernel

    for W in available_widths():
        k = load_kernel(W)
        assert k.horner.shape == (W, 8) and k.theta.size == M.NTHETA
        d = np.linspace(-W / 2 + 1e-6, W / 2 - 1e-6, 2001)
        ref = k.phi(d)
        assert np.abs(M.horner_eval(k.horner, W, d) - ref).max() <= 1e-3 * np.abs(ref).max()
        # the Horner form keeps the trained network's accuracy on the held-out sets
        ev = k.meta["eval_2d"]
        assert ev["rel_l2_learned_horner"] <= 1.05 * ev["rel_l2_learned"] < ev["rel_l2_es"]


def test_width_search_record():
    """The committed width search: the learned kernel meets each epsilon at a
    width no larger than ES needs, and errors fall with W up to the FP32 floor."""
    import json
    import os

    from cugridder_b200.learn.model import KERNEL_DIR

    p = os.path.join(KERNEL_DIR, "wsearch_2048_10M.json")
    if not os.path.exists(p):
        pytest.skip("no width search recorded")
    with open(p) as f:
        ws = json.load(f)
    for eps, best in ws["smallest_W"].items():
        if best["es"] is not None:
            assert best["learned"] is not None and best["learned"] <= best["es"]
    for r in ws["results"]:
        if r["kernel"] == "learned":
            es = [q for q in ws["results"] if q["kernel"] == "es" and q["W"] == r["W"]][0]
            assert r["err_ms2dirty"] < es["err_ms2dirty"] and r["err_dirty2ms"] < es["err_dirty2ms"]
