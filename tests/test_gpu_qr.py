"""FP64 DMMA GEMM and the Householder QR (client.cpp:417-445) on the GPU
against LAPACK / numpy in FP64."""
import numpy as np
import pytest
import scipy.linalg.lapack as lapack

from gpu_util import context

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return context()


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (129, 65, 17), (32, 1000, 200000), (1000, 1000, 1000), (7, 300, 5)])
def test_dgemm_matches_numpy(ctx, ta, tb, M, N, K):
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    opA = rng.standard_normal((M, K))
    opB = rng.standard_normal((K, N))
    C0 = rng.standard_normal((M, N))
    # column-major storage: a column-major X is the row-major tensor X^T
    Acm = opA.T if ta else opA               # the stored (column-major) A
    Bcm = opB.T if tb else opB
    tA = ctx._dev(np.ascontiguousarray(Acm.T))
    tB = ctx._dev(np.ascontiguousarray(Bcm.T))
    tC = ctx._dev(np.ascontiguousarray(C0.T))
    out = ctx.dgemm(ta, tb, tA, tB, alpha=1.5, beta=-0.5, C=tC).cpu().numpy().T
    ref = 1.5 * opA @ opB - 0.5 * C0
    assert np.max(np.abs(out - ref)) < 1e-13 * K ** 0.5 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("n,m", [(1000, 100), (4099, 257), (20000, 64), (300, 33)])
def test_local_qr_matches_lapack(ctx, n, m):
    rng = np.random.default_rng(n + m)
    X = rng.standard_normal((m, n))          # participant block, row-major m x n
    t = ctx._dev(X.copy())
    rt = ctx.local_qr_reduction(t, compute_q=True).cpu().numpy()
    Qt = t.cpu().numpy()                     # Q^T, m x n
    qr, tau, _, _ = lapack.dgeqrf(np.asfortranarray(X.T))
    R = np.triu(qr[:m])
    # same Householder convention (dlarfg) as LAPACK: same signs
    assert np.max(np.abs(rt - R.T)) < 1e-12 * np.abs(R).max()
    assert np.allclose(np.tril(rt), rt)
    assert np.max(np.abs(Qt @ Qt.T - np.eye(m))) < 1e-13 * n ** 0.5
    assert np.max(np.abs(rt @ Qt - X)) < 1e-12 * np.abs(X).max() * m ** 0.5


def test_local_qr_rejects_short_blocks(ctx):
    import excalibur_b200 as eb
    t = ctx._dev(np.ones((10, 10)))
    with pytest.raises(eb.BBTError):
        ctx.local_qr_reduction(t)
