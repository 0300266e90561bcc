"""FP64-accurate GEMM from exact int8 slices on the tensor cores (the Ozaki
scheme, csrc/ozaki.cu) against an extended-precision product, next to the
DMMA FP64 GEMM on the same inputs."""
import numpy as np
import pytest

from gpu_util import context

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return context()


def operands(rng, ta, tb, M, N, K):
    """op(A) M x K, op(B) K x N with rows/columns scaled over six decades,
    and the tensors holding A, B in the library's column-major convention."""
    opA = rng.standard_normal((M, K)) * 10.0 ** rng.uniform(-3, 3, (M, 1))
    opB = rng.standard_normal((K, N)) * 10.0 ** rng.uniform(-3, 3, (1, N))
    A = opA.T if ta else opA           # the stored matrix (column-major)
    B = opB.T if tb else opB
    return opA, opB, np.ascontiguousarray(A.T), np.ascontiguousarray(B.T)


@pytest.mark.parametrize("ta,tb,M,N,K,beta", [
    (0, 0, 300, 200, 3000, 0.0),
    (1, 0, 256, 256, 20000, 0.0),      # Gram-like: A^T A shapes
    (0, 0, 4000, 160, 512, 1.0),       # triangular-solve update: C -= A1 R12
    (0, 1, 130, 70, 100, 0.5),         # tails in M, N and K
    (1, 1, 200, 96, 777, -1.0),
])
def test_ozaki_gemm_accuracy(ctx, ta, tb, M, N, K, beta):
    rng = np.random.default_rng(M + N + K)
    opA, opB, At, Bt = operands(rng, ta, tb, M, N, K)
    C0 = rng.standard_normal((M, N))
    alpha = -1.0 if beta == 1.0 else 1.25
    exact = alpha * (opA.astype(np.longdouble) @ opB.astype(np.longdouble)) + beta * C0.astype(np.longdouble)
    bound = np.abs(opA) @ np.abs(opB) * abs(alpha) + abs(beta) * np.abs(C0)
    dev = lambda x: ctx._dev(np.ascontiguousarray(x))
    got = ctx.dgemm_ozaki(ta, tb, dev(At), dev(Bt), alpha, beta, dev(C0.T)).cpu().numpy().T
    dm = ctx.dgemm(ta, tb, dev(At), dev(Bt), alpha, beta, dev(C0.T)).cpu().numpy().T
    err_oz = np.max(np.abs(got - exact) / bound)
    err_dm = np.max(np.abs(dm - exact) / bound)
    print(f"M={M} N={N} K={K}: ozaki {err_oz:.2e}, dmma {err_dm:.2e} (relative to |A||B|)")
    assert err_oz < 2.0 ** -50, err_oz
    assert err_oz < 8 * max(err_dm, 2.0 ** -53), (err_oz, err_dm)


def test_ozaki_upper_triangle(ctx):
    """upper: the tiles on or above the diagonal are computed, the others
    keep C's old values."""
    rng = np.random.default_rng(3)
    K, M = 5000, 300
    A = rng.standard_normal((K, M))                   # column-major M x K stored transposed: op(A) = A^T
    C = np.full((M, M), 7.0)
    got = ctx.dgemm_ozaki(1, 0, ctx._dev(A.T.copy()), ctx._dev(A.T.copy()), 1.0, 0.0, ctx._dev(C.T.copy()),
                          upper=True).cpu().numpy().T
    ref = (A.T.astype(np.longdouble) @ A.astype(np.longdouble))
    iu = np.triu_indices(M)
    assert np.max(np.abs(got[iu] - ref[iu]) / (np.abs(A).T @ np.abs(A))[iu]) < 2.0 ** -50
    # tiles strictly below the diagonal (128-row x 64-column tiles) are untouched
    for i in range(M):
        for j in range(M):
            if (i // 128) * 128 >= (j // 64) * 64 + 64:
                assert got[i, j] == 7.0
