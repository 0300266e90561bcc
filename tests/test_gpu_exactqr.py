"""The exact-Gram local QR (precision mode 2, csrc/exactqr.cu): R against
LAPACK's dgeqrf (row signs included), the implicit Q = A_int R_p^-1 W applied
by exact products orthonormal to FP64 level, and Q R = A, for blocks of
condition number up to 1e6."""
import numpy as np
import pytest

from gpu_util import context

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return context()


def block(m, n, cond, seed):
    rng = np.random.default_rng(seed)
    U, _ = np.linalg.qr(rng.standard_normal((n, m)))
    V, _ = np.linalg.qr(rng.standard_normal((m, m)))
    s = np.geomspace(1.0, 1.0 / cond, m)
    return np.ascontiguousarray(((U * s) @ V.T).T)   # X = A^T, row-major m x n


@pytest.mark.parametrize("m,n,cond", [(64, 3000, 1e2), (300, 60000, 1e6), (500, 20000, 1e4)])
def test_exact_qr_against_lapack(ctx, m, n, cond):
    X = block(m, n, cond, m + n)
    Xd = ctx._dev(X)
    Rt, Wt, Rpt, sc = ctx.exact_local_qr(Xd)
    R = Rt.cpu().numpy().T
    assert np.array_equal(Xd.cpu().numpy(), X)   # the block is kept
    assert np.all(np.tril(R, -1) == 0.0)
    Rl = np.linalg.qr(X.T, mode="r")   # dgeqrf
    assert np.all(np.sign(np.diag(R)) == np.sign(np.diag(Rl)))
    assert np.max(np.abs(R - Rl)) / np.max(np.abs(Rl)) < 1e-15 * cond * 10
    sl = np.linalg.svd(X, compute_uv=False)
    assert np.max(np.abs(np.linalg.svd(R, compute_uv=False) - sl) / sl) < 1e-15 * cond * 10
    # Q = A_int R_p^-1 W, applied to the identity
    Q = ctx.exact_apply_q(Xd, sc, Rpt, Wt).cpu().numpy().T   # n x m
    assert np.max(np.abs(Q.T @ Q - np.eye(m))) < 1e-13
    assert np.linalg.norm(Q @ R - X.T) / np.linalg.norm(X) < 1e-14   # FP64 evaluation of Q @ R included
    # against LAPACK's Q with the same row signs
    Ql = np.linalg.qr(X.T)[0]
    assert np.max(np.abs(Q - Ql)) < 1e-15 * cond * 100
