"""CPU checks of the MLP restatement the GPU kernels are tested against:
its analytic gradient against central finite differences, and its features
against a direct computation."""
import numpy as np

from oracle import mlp


def test_numpy_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    theta = mlp.init(1) + 0.1 * rng.standard_normal(mlp.NPARAM)
    X = rng.standard_normal((64, mlp.F)) * 0.5
    y = rng.uniform(-30, 0, 64) / 8.0
    loss, g = mlp.loss_grad(theta, X, y)
    idx = rng.choice(mlp.NPARAM, 80, replace=False)
    h = 1e-6
    for q in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[q] += h
        tm[q] -= h
        fd = (mlp.loss_grad(tp, X, y)[0] - mlp.loss_grad(tm, X, y)[0]) / (2 * h)
        assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(g[q])), (q, fd, g[q])


def test_features():
    rng = np.random.default_rng(4)
    a, b = rng.uniform(0.5, 2.0, 50), rng.uniform(-1, 1, 49)
    X, g = mlp.features(a, b)
    assert X.shape == (50, mlp.F)
    gg = max(abs(a[i]) + max(abs(b[i - 1]) if i > 0 else 0, abs(b[i]) if i < 49 else 0) for i in range(50))
    assert g == gg
    assert np.allclose(X[:, 0], np.log2(np.linalg.norm(a) / g) / 16)
    assert np.allclose(X[:, 6], (np.arange(50) + 0.5) / 50)
    assert np.all(X[:, 2:5] <= 0)   # max|a|, max|b|, min|a| never exceed g
