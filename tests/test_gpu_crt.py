"""Exact integer products on the int8 tensor cores by the Chinese remainder
theorem (csrc/crt.cu): the Gram matrix as a double-double against the exact
integer product of the same rounded rows, and the FP64 product against the
exact value."""
from fractions import Fraction

import numpy as np
import pytest

from gpu_util import context

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return context()


def row_integers(X, bits):
    """The rounding the library applies: s_i = 2^(e+1) with max|x| in
    [2^(e-1), 2^e), t = rint(x 2^(bits-1) / s_i)."""
    mx = np.abs(X).max(axis=1)
    e = np.frexp(mx)[1]
    s = np.ldexp(1.0, e + 1)
    t = np.rint(X * (np.ldexp(1.0, bits - 1) / s)[:, None])
    return t, s


def exact_product(ta, tb):
    """ta @ tb.T exactly (Python ints), integer-valued float inputs < 2^52, via
    17-bit pieces and int64 products."""
    def pieces(t):
        t = t.astype(np.int64)
        sg = np.sign(t)
        a = np.abs(t)
        return [sg * ((a >> (17 * k)) & 0x1FFFF) for k in range(3)]
    pa, pb = pieces(ta), pieces(tb)
    out = np.zeros((ta.shape[0], tb.shape[0]), dtype=object)
    for u in range(3):
        for v in range(3):
            out += (pa[u] @ pb[v].T).astype(object) * (1 << (17 * (u + v)))
    return out


@pytest.mark.parametrize("m,n", [(64, 3000), (200, 150_000), (300, 1000)])
def test_gram_dd_is_exact(ctx, m, n):
    rng = np.random.default_rng(m + n)
    X = rng.standard_normal((m, n)) * np.exp2(rng.integers(-20, 20, (m, 1)))
    X[:, ::7] *= 1e-9   # small entries lose bits only relative to their row's maximum
    Gh, Gl = ctx.gram_dd(ctx._dev(X))
    Gh, Gl = Gh.cpu().numpy().T, Gl.cpu().numpy().T   # column-major storage
    t, s = row_integers(X, 53)
    T = exact_product(t, t)
    worst = Fraction(0)
    for i in range(0, m, max(1, m // 40)):
        for j in range(i, m, max(1, m // 40)):
            exact = Fraction(int(T[i, j])) * Fraction(s[i]) * Fraction(s[j]) / 2 ** 104
            got = Fraction(Gh[i, j]) + Fraction(Gl[i, j])
            scale = Fraction(s[i]) * Fraction(s[j]) * n
            worst = max(worst, abs(got - exact) / scale)
    assert worst < Fraction(1, 2 ** 100), float(worst)


@pytest.mark.parametrize("M,N,K", [(300, 500, 1000), (257, 129, 70_000), (1000, 1000, 4096)])
def test_dgemm_crt_accuracy(ctx, M, N, K):
    rng = np.random.default_rng(M * N + K)
    A = rng.standard_normal((M, K))   # rows of A^T: column-major K x M
    B = rng.standard_normal((N, K))
    C0 = rng.standard_normal((N, M))
    C = ctx.dgemm_crt(ctx._dev(A), ctx._dev(B), alpha=-1.0, beta=1.0, C=ctx._dev(C0.copy())).cpu().numpy()
    ta, sa = row_integers(A, 53)
    tb, sb = row_integers(B, 53)
    # reference from the exact product of the rounded rows, rounded once
    T = exact_product(ta, tb) if M * N * K <= 3e8 else None
    if T is not None:
        ref = np.array([[float(Fraction(int(T[i, j])) * Fraction(sa[i] * sb[j]) / 2 ** 104) for j in range(N)]
                        for i in range(M)])
        err = np.abs(C - (C0 - ref.T)) / (np.abs(A).max(1)[None, :] * np.abs(B).max(1)[:, None] * K)
        assert err.max() < 2.0 ** -50
    ref_ld = C0.astype(np.longdouble) - (B.astype(np.longdouble) @ A.astype(np.longdouble).T)
    # against the unrounded FP64 inputs: the 53-bit row rounding, DGEMM-level
    assert np.max(np.abs(C - ref_ld.astype(np.float64))) / np.max(np.abs(ref_ld)) < 1e-14
