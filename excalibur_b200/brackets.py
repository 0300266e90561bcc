"""Learned bisection brackets: training-data generation and training on the
GPU through the library's own kernels (mlp.cu), and the trained parameters.

    python -m excalibur_b200.brackets --out excalibur_b200/data/bracket_mlp.npz

builds bidiagonals with the pipeline's own Householder bidiagonalisation
(bbt_gebrd) of X = U diag(s) V^T (Haar U, V) for the spectrum families below,
takes their singular values from the plain bisection (bbt_bisection_singular
values), and fits the MLP (bbt_mlp_grad + bbt_mlp_adam).  The committed file
is loaded by ``load_model``; ``Context.set_bracket_model`` switches it on.

Families (sizes drawn from `sizes`):
  clustered  -- clusters of 16 values at relative spacing 1e-10, centres
                log-uniform in [1e-8, 1] (the 8192 x 8192 stress family);
  geometric  -- s from 1 down to 10^-U[3, 8], geometric (the tall-skinny
                family's spectrum).
"""
import argparse
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(HERE, "data", "bracket_mlp.npz")
Z = 3.0   # bracket half-width in units of the predicted spread


def spectrum(family, n, rng):
    if family == "clustered":
        c = np.exp(rng.uniform(np.log(1e-8), 0.0, max(1, n // 16)))
        s = np.concatenate([ci * (1.0 + 1e-10 * np.arange(16)) for ci in c])[:n]
        if len(s) < n:
            s = np.concatenate([s, np.exp(rng.uniform(np.log(1e-8), 0.0, n - len(s)))])
    elif family == "geometric":
        s = np.geomspace(1.0, 10.0 ** -rng.uniform(3.0, 8.0), n)
    else:
        raise ValueError(family)
    return np.sort(s)[::-1].copy()


def make_bidiagonal(ctx, family, n, seed):
    """(a, b) of X = U diag(s) V^T by the library's Householder
    bidiagonalisation; device tensors."""
    torch = ctx.torch
    rng = np.random.default_rng(seed)
    s = spectrum(family, n, rng)
    dev = f"cuda:{ctx.device}"
    g = torch.Generator(device=dev).manual_seed(int(seed))

    def haar(m):
        q, r = torch.linalg.qr(torch.randn(m, m, generator=g, device=dev, dtype=torch.float64))
        return q * torch.sign(torch.diagonal(r))

    X = (haar(n) * torch.as_tensor(s, device=dev)) @ haar(n).T
    a, b = ctx.gebrd(X.T.contiguous())   # column-major X
    return a, b


def samples(ctx, a, b):
    """(features, log2(sigma_j / g)) for every singular value found by the
    plain bisection (the targets are the method's own outputs)."""
    torch = ctx.torch
    k = a.numel()
    sig = ctx.bidiagonal_singular_values(a, b)
    cnt = sig.numel()
    if cnt == 0:
        return None
    X = ctx.mlp_features(a, b, cnt)
    g = float(np.max(np.abs(a.cpu().numpy()) + np.maximum(
        np.abs(np.concatenate([[0.0], b.cpu().numpy()[: k - 1]])),
        np.abs(np.concatenate([b.cpu().numpy()[: k - 1], [0.0]])))))
    y = torch.log2(torch.clamp(sig, min=1e-300) / g)
    return X, y


def build_dataset(ctx, count, sizes, families, seed=0, log=None):
    Xs, ys = [], []
    rng = np.random.default_rng(seed)
    for i in range(count):
        fam = families[i % len(families)]
        n = int(rng.choice(sizes))
        a, b = make_bidiagonal(ctx, fam, n, seed * 1000003 + i)
        smp = samples(ctx, a, b)
        if smp is not None:
            Xs.append(smp[0])
            ys.append(smp[1])
        if log and (i + 1) % 100 == 0:
            log(f"  {i + 1}/{count} bidiagonals")
    torch = ctx.torch
    return torch.cat(Xs), torch.cat(ys)


def init_params(seed=0):
    """Glorot-uniform weights, zero biases; the spread output starts at
    log(2), the centre at -1."""
    F, H = 10, 32
    rng = np.random.default_rng(seed)
    out = []
    for name, shp in [("W1", (H, F)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (2, H)), ("b3", (2,))]:
        if name.startswith("W"):
            lim = np.sqrt(6.0 / (shp[0] + shp[1]))
            out.append(rng.uniform(-lim, lim, shp).ravel())
        elif name == "b3":
            out.append(np.array([-1.0, np.log(2.0)]))
        else:
            out.append(np.zeros(shp))
    return np.concatenate(out)


def fit(ctx, X, y, steps=3000, batch=4096, lr=2e-3, seed=0, theta0=None, log=None):
    """Adam on minibatches; every step is one gradient kernel and one Adam
    kernel on the device.  Returns (theta as numpy, loss history)."""
    torch = ctx.torch
    dev = X.device
    theta = torch.as_tensor(init_params(seed) if theta0 is None else theta0, device=dev, dtype=torch.float64)
    m = torch.zeros_like(theta)
    v = torch.zeros_like(theta)
    grad = torch.zeros_like(theta)
    loss = torch.zeros(1, device=dev, dtype=torch.float64)
    g = torch.Generator(device=dev).manual_seed(seed)
    hist = []
    N = X.shape[0]
    for t in range(1, steps + 1):
        idx = torch.randint(0, N, (min(batch, N),), generator=g, device=dev)
        Xb, yb = X[idx].contiguous(), y[idx].contiguous()
        ctx.mlp_grad(Xb, yb, theta, grad, loss)
        ctx.mlp_adam(theta, grad, m, v, lr * (0.1 ** (t / steps)), t)
        if t % 50 == 0 or t == 1:
            hist.append((t, float(loss)))
            if log and t % 5000 == 0:
                log(f"  step {t}: loss {hist[-1][1]:.4f}")
    return theta.cpu().numpy(), hist


def load_model(path=DEFAULT_MODEL):
    """(theta, z) of the committed model."""
    d = np.load(path)
    return d["theta"], float(d["z"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_MODEL)
    ap.add_argument("--count", type=int, default=1200)
    ap.add_argument("--sizes", default="256,384,512,768,1024")
    ap.add_argument("--steps", type=int, default=60000)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    import excalibur_b200 as eb
    ctx = eb.Context(0)
    t0 = time.time()
    sizes = [int(x) for x in args.sizes.split(",")]
    X, y = build_dataset(ctx, args.count, sizes, ["clustered", "geometric"], seed=args.seed, log=print)
    t1 = time.time()
    print(f"dataset: {X.shape[0]} samples from {args.count} bidiagonals in {t1 - t0:.1f} s")
    theta, hist = fit(ctx, X, y, steps=args.steps, seed=args.seed, log=print)
    print(f"trained {args.steps} steps in {time.time() - t1:.1f} s; loss {hist[0][1]:.4f} -> {hist[-1][1]:.4f}")
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    np.savez(args.out, theta=theta, z=Z, loss=np.array(hist), count=args.count, sizes=np.array(sizes),
             families=np.array(["clustered", "geometric"]), samples=X.shape[0])
    print("wrote", args.out)


if __name__ == "__main__":
    main()
