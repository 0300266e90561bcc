"""ORACLE -- test infrastructure, not product code.

numpy restatement of the learned-bracket MLP (the library's mlp.cu): the
features of a bidiagonal, the forward pass, the Gaussian negative
log-likelihood and its exact gradient.  The reference has no learned part;
this is the CPU check of the library's own CUDA forward/backward kernels.
Parameter layout (flat float64): W1 (H x F row-major), b1 (H), W2 (H x H),
b2 (H), W3 (2 x H), b3 (2).
"""
import numpy as np

F, H = 10, 32
SIZES = [("W1", (H, F)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (2, H)), ("b3", (2,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(theta):
    out, o = {}, 0
    for name, shp in SIZES:
        n = int(np.prod(shp))
        out[name] = theta[o:o + n].reshape(shp)
        o += n
    return out


def pack(parts):
    return np.concatenate([parts[name].ravel() for name, _ in SIZES])


def init(seed=0):
    """Glorot-uniform weights, zero biases; the spread output starts at
    log(2) (a two-octave bracket)."""
    rng = np.random.default_rng(seed)
    parts = {}
    for name, shp in SIZES:
        if name.startswith("W"):
            lim = np.sqrt(6.0 / (shp[0] + shp[1]))
            parts[name] = rng.uniform(-lim, lim, shp)
        else:
            parts[name] = np.zeros(shp)
    parts["b3"] = np.array([-1.0, np.log(2.0)])
    return pack(parts)


def _clip_log(r):
    with np.errstate(divide="ignore"):
        l = np.where(r > 0, np.log2(np.where(r > 0, r, 1.0)), -64.0)
    return np.clip(l, -64.0, 16.0) / 16.0


def summary(a, b):
    a, b = np.abs(np.asarray(a, float)), np.abs(np.asarray(b, float))
    k = len(a)
    bl = np.concatenate([[0.0], b[: k - 1]]) if k > 1 else np.zeros(1)
    br = np.concatenate([b[: k - 1], [0.0]]) if k > 1 else np.zeros(1)
    g = np.max(a + np.maximum(bl, br))
    bb = b[: k - 1]
    return (np.linalg.norm(a), np.linalg.norm(bb) if k > 1 else 0.0, a.max(),
            bb.max() if k > 1 else 0.0, a.min(), g)


def features(a, b, count=None):
    """(count x F) features of the j-th largest value, j = 0 .. count-1."""
    k = len(a)
    count = k if count is None else count
    s = summary(a, b)
    g = s[5] if s[5] > 0 else 1.0
    t = (np.arange(count) + 0.5) / k
    glob = [_clip_log(np.float64(v) / g) for v in s[:5]] + [np.log2(k) / 16.0]
    X = np.empty((count, F))
    X[:, :6] = glob
    X[:, 6], X[:, 7], X[:, 8], X[:, 9] = t, t * t, np.sqrt(t), np.log2(t) / 16.0
    return X, g


def forward(theta, X):
    p = unpack(theta)
    h1 = np.tanh(X @ p["W1"].T + p["b1"])
    h2 = np.tanh(h1 @ p["W2"].T + p["b2"])
    return h2 @ p["W3"].T + p["b3"], (h1, h2)


def loss_grad(theta, X, y):
    """Mean Gaussian NLL 0.5 ((y - mu) e^-ell)^2 + ell and its gradient."""
    p = unpack(theta)
    out, (h1, h2) = forward(theta, X)
    mu, ell = out[:, 0], out[:, 1]
    r = y - mu
    e2 = np.exp(-2.0 * ell)
    loss = np.mean(0.5 * r * r * e2 + ell)
    B = len(y)
    d3 = np.stack([-r * e2, 1.0 - r * r * e2], axis=1) / B
    g = {"W3": d3.T @ h2, "b3": d3.sum(0)}
    d2 = (d3 @ p["W3"]) * (1.0 - h2 * h2)
    g["W2"], g["b2"] = d2.T @ h1, d2.sum(0)
    d1 = (d2 @ p["W2"]) * (1.0 - h1 * h1)
    g["W1"], g["b1"] = d1.T @ X, d1.sum(0)
    return loss, pack(g)
