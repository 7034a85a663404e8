"""The learned kernel family, its FP64 evaluation, the Horner fit and the
artifact format.

    phi(d) = exp(beta0 * (sqrt(1 - t^2) - 1) + net(2 t^2 - 1)),  t = 2 d / W,  |t| < 1

``net`` is a 1-32-32-1 tanh MLP.  beta0 = 2.30 W, the ES shape parameter that
the reference's setup_conv_opts picks (conv_interp_invoker.cu:49-119), so a
zero network is the ES kernel exp(beta0 sqrt(1 - t^2)) up to a constant
factor, and training learns a log-domain correction.  theta layout (1153
floats): W1[32], b1[32], W2[32][32] (row = output unit), b2[32], w3[32], b3.

Horner form used by the gridder: W segments; segment i covers
d in [i - W/2, i + 1 - W/2) and is sum_n a[i][n] s^n with
s = 2 (d + W/2 - i) - 1 in [-1, 1), degree 7.
"""
import json
import os

import numpy as np

H = 32
NTHETA = H + H + H * H + H + H + 1
DEG = 7
FORMAT = "cugridder-b200 learned kernel v1"
KERNEL_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "kernels")


def beta0_for(W):
    """ES shape of the reference's setup_conv_opts for sigma = 2."""
    b = {2: 2.20, 3: 2.26, 4: 2.38}.get(W, 2.30)
    return b * W


def split_theta(th):
    th = np.asarray(th, dtype=np.float64)
    W1, b1 = th[:H], th[H:2 * H]
    W2 = th[2 * H:2 * H + H * H].reshape(H, H)
    o = 2 * H + H * H
    b2, w3, b3 = th[o:o + H], th[o + H:o + 2 * H], th[o + 2 * H]
    return W1, b1, W2, b2, w3, b3


def init_theta(seed=0):
    """Random hidden layers, zero output layer: the initial kernel is ES."""
    rng = np.random.Generator(np.random.PCG64(seed))
    th = np.zeros(NTHETA, dtype=np.float64)
    th[:H] = rng.normal(0.0, 1.5, H)                                    # W1
    th[H:2 * H] = rng.uniform(-1.0, 1.0, H)                             # b1
    th[2 * H:2 * H + H * H] = rng.normal(0.0, 1.0 / np.sqrt(H), H * H)  # W2
    return th


def net_np(th, x):
    W1, b1, W2, b2, w3, b3 = split_theta(th)
    x = np.asarray(x, dtype=np.float64)[..., None]
    h1 = np.tanh(x * W1 + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h2 @ w3 + b3


def phi_np(th, beta0, W, d):
    """FP64 kernel value at distance d (grid cells); 0 outside |d| < W/2."""
    d = np.asarray(d, dtype=np.float64)
    t2 = (2.0 * d / W) ** 2
    inside = t2 < 1.0
    t2c = np.where(inside, t2, 0.0)
    v = np.exp(beta0 * (np.sqrt(1.0 - t2c) - 1.0) + net_np(th, 2.0 * t2c - 1.0))
    return np.where(inside, v, 0.0)


def horner_fit(fun, W, deg=DEG, nodes=96):
    """Least-squares fit of each unit segment of fun(d), d in [-W/2, W/2], by a
    degree-`deg` polynomial in s = 2 (d + W/2 - i) - 1 on Chebyshev nodes;
    returns coefficients [W, 8] (monomials in s, zero-padded to 8)."""
    k = np.arange(nodes)
    s = np.cos(np.pi * (k + 0.5) / nodes)  # Chebyshev points of the first kind
    coef = np.zeros((W, 8))
    for i in range(W):
        d = (s + 1.0) / 2.0 + i - W / 2.0
        c = np.polynomial.chebyshev.chebfit(s, fun(d), deg)
        coef[i, :deg + 1] = np.polynomial.chebyshev.cheb2poly(c)
    return coef


def horner_eval(coef, W, d):
    d = np.asarray(d, dtype=np.float64)
    u = d + W / 2.0
    s = np.floor(u).astype(np.int64)
    ok = (s >= 0) & (s < W)
    sc = np.clip(s, 0, W - 1)
    t = 2.0 * (u - sc) - 1.0
    v = np.zeros_like(d)
    for n in range(coef.shape[1] - 1, -1, -1):
        v = v * t + coef[sc, n]
    return np.where(ok, v, 0.0)


def es_horner(W, beta=None):
    """Horner table of the ES kernel exp(beta (sqrt(1 - t^2) - 1)) (the zero
    network), for comparisons at equal evaluation cost."""
    b0 = beta0_for(W) if beta is None else beta
    zero = np.zeros(NTHETA)
    return horner_fit(lambda d: phi_np(zero, b0, W, d), W)


class LearnedKernel:
    def __init__(self, W, beta0, theta, horner, meta=None):
        self.W = int(W)
        self.beta0 = float(beta0)
        self.theta = np.asarray(theta, dtype=np.float64)
        self.horner = np.asarray(horner, dtype=np.float64).reshape(self.W, 8)
        self.meta = dict(meta or {})

    def phi(self, d):
        return phi_np(self.theta, self.beta0, self.W, d)

    def to_json(self):
        return {
            "format": FORMAT, "W": self.W, "beta0": self.beta0,
            "theta": [float(v) for v in self.theta],
            "horner": [[float(v) for v in row] for row in self.horner],
            **self.meta,
        }

    def save(self, path):
        with open(path, "w") as f:
            json.dump(self.to_json(), f, indent=1)
        np.asarray(self.theta, dtype="<f8").tofile(os.path.splitext(path)[0] + ".theta.bin")

    @classmethod
    def from_json(cls, d):
        if d.get("format") != FORMAT:
            raise ValueError("not a %s artifact" % FORMAT)
        meta = {k: v for k, v in d.items() if k not in ("format", "W", "beta0", "theta", "horner")}
        return cls(d["W"], d["beta0"], d["theta"], d["horner"], meta)


def kernel_path(W, directory=None):
    return os.path.join(directory or KERNEL_DIR, "learned_W%d.json" % int(W))


def available_widths(directory=None):
    d = directory or KERNEL_DIR
    if not os.path.isdir(d):
        return []
    out = []
    for fn in os.listdir(d):
        if fn.startswith("learned_W") and fn.endswith(".json"):
            out.append(int(fn[len("learned_W"):-len(".json")]))
    return sorted(out)


def load_kernel(W, directory=None):
    with open(kernel_path(W, directory)) as f:
        return LearnedKernel.from_json(json.load(f))


def smallest_width(eps, directory=None):
    """The learned kernel at the smallest width that met eps in the committed
    width search (kernels/wsearch_2048_10M.json), or None when none did."""
    import json

    p = os.path.join(directory or KERNEL_DIR, "wsearch_2048_10M.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        best = json.load(f).get("smallest_W", {})
    W = (best.get("%g" % eps) or {}).get("learned")
    if W is None or W not in available_widths(directory):
        return None
    return load_kernel(W, directory)
