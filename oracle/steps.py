"""ORACLE — test infrastructure, not product code.

Pure-Python restatement of the reference's per-step helpers of the twisted
factorisation and its small vector helpers (Excalibur src/bbtsvd.cpp), for
small cases.  Python floats are IEEE doubles with every operation rounded
on its own, as in the reference's no-FMA build, so the recurrences reproduce
the reference bit for bit; the vectors it normalises with BLAS dnrm2 are
normalised here by the scaled sum of squares (equal to rounding)."""
import math


def ldl_decomposition(a, b):
    """LDL^T of B^T B (bbtsvd.cpp:54-63): l (n-1), d (n)."""
    n = len(a)
    d = [a[0] * a[0]] + [0.0] * (n - 1)
    l = [0.0] * max(n - 1, 0)
    for i in range(1, n):
        ab = a[i - 1] * b[i - 1]
        l[i - 1] = ab / d[i - 1]
        d[i] = (a[i] * a[i] + b[i - 1] * b[i - 1]) - (ab * ab) / d[i - 1]
    return l, d


def dstqds(l, d, tau):
    """Stationary qd transform of L D L^T - tau I (bbtsvd.cpp:73-81)."""
    n = len(d)
    s = [0.0] * n
    lp = [0.0] * max(n - 1, 0)
    dp = [0.0] * n
    s[0] = -tau
    for i in range(n - 1):
        dp[i] = d[i] + s[i]
        lp[i] = (d[i] * l[i]) / dp[i]
        s[i + 1] = (lp[i] * l[i]) * s[i] - tau
    dp[n - 1] = d[n - 1] + s[n - 1]
    return lp, dp, s


def dpqds(l, d, tau):
    """Progressive qd transform (bbtsvd.cpp:83-91)."""
    n = len(d)
    p = [0.0] * n
    rp = [0.0] * n
    up = [0.0] * max(n - 1, 0)
    p[n - 1] = d[n - 1] - tau
    for i in range(n - 2, -1, -1):
        rp[i + 1] = d[i] * (l[i] * l[i]) + p[i + 1]
        up[i] = (l[i] * d[i]) / rp[i + 1]
        p[i] = (p[i + 1] * d[i]) / rp[i + 1] - tau
    rp[0] = p[0]
    return up, rp, p


def _norm(x):
    scale, ssq = 0.0, 1.0
    for v in x:
        v = abs(v)
        if v != 0.0:
            if scale < v:
                r = scale / v
                ssq = 1.0 + (ssq * r) * r
                scale = v
            else:
                r = v / scale
                ssq = ssq + r * r
    return scale * math.sqrt(ssq)


def inverse_iteration(n, k, l, u):
    """v[k] = 1, backward with l, forward with u, normalised (bbtsvd.cpp:65-71)."""
    v = [0.0] * n
    v[k] = 1.0
    for i in range(k - 1, -1, -1):
        v[i] = -l[i] * v[i + 1]
    for i in range(k + 1, n):
        v[i] = -u[i - 1] * v[i - 1]
    r = 1.0 / _norm(v)
    return [x * r for x in v]


def generate_house(x):
    """Householder vector of x (bbtsvd.cpp:149-164): (x', beta)."""
    x = list(x)
    n = len(x)
    sigma = 0.0
    for i in range(1, n):
        sigma += x[i] * x[i]
    x0 = x[0]
    x[0] = 1.0
    if sigma == 0.0 and x0 >= 0.0:
        return x, 0.0
    if sigma == 0.0 and x0 < 0.0:
        return x, 2.0
    mu = math.sqrt(x0 * x0 + sigma)
    h = x0 - mu if x0 <= 0.0 else -sigma / (x0 + mu)
    x[0] = h
    beta = (2.0 * (h * h)) / (sigma + h * h)
    r = 1.0 / h
    return [v * r for v in x], beta


def mmap_drot(x, y, c, s):
    """(x, y) <- (x c + y s, x (-s) + y c) elementwise (bbtsvd.cpp:970-978)."""
    return [xi * c + yi * s for xi, yi in zip(x, y)], [xi * -s + yi * c for xi, yi in zip(x, y)]
