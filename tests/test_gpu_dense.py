"""bbt_svd_dense: Ralha bidiagonalisation + bisection + twisted vectors +
back-transforms on one dense matrix (the chain of client.cpp:801-1176),
against LAPACK FP64."""
import numpy as np
import pytest

from gpu_util import context, gap_groups, subspace_angle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return context()


def haar(rng, n):
    q, r = np.linalg.qr(rng.standard_normal((n, n)))
    return q * np.sign(np.diag(r))


def clustered_spectrum(rng, clusters, size, gap=1e-10, lo=1e-8, hi=1.0):
    """The 8192^2 stress family at any size: clusters of `size` values at
    relative spacing `gap`, centres log-uniform in [lo, hi]."""
    c = np.exp(rng.uniform(np.log(lo), np.log(hi), clusters))
    s = np.concatenate([ci * (1.0 + gap * np.arange(size)) for ci in c])
    return np.sort(s)[::-1]


@pytest.mark.parametrize("m", [64, 300])
def test_dense_svd_random(ctx, m):
    rng = np.random.default_rng(m)
    X = rng.standard_normal((m, m))
    s, U, VT = ctx.svd_dense(ctx._dev(X.copy()))
    s, U, VT = s.cpu().numpy(), U.cpu().numpy(), VT.cpu().numpy()
    Ul, sl, Vl = np.linalg.svd(X)
    assert len(s) == m
    assert np.max(np.abs(s - sl) / sl) < 1e-10
    assert np.max(np.abs(U @ np.diag(s) @ VT - X)) < 1e-12 * np.abs(X).max() * m
    for grp in gap_groups(sl):
        assert subspace_angle(U[:, grp], Ul[:, grp]) < 1e-8
        assert subspace_angle(VT[grp].T, Vl[grp].T) < 1e-8


def test_dense_svd_geometric_top_k(ctx):
    rng = np.random.default_rng(5)
    m = 256
    sv = np.geomspace(1.0, 1e-6, m)
    X = haar(rng, m) @ np.diag(sv) @ haar(rng, m).T
    s, U, VT = ctx.svd_dense(ctx._dev(X.copy()), top_k=20)
    s = s.cpu().numpy()
    sl = np.linalg.svd(X, compute_uv=False)
    assert len(s) == 20
    assert np.max(np.abs(s - sl[:20]) / sl[:20]) < 1e-10


def test_dense_svd_clustered_values(ctx):
    """Clustered spectrum (the 8192^2 stress family at m = 256): singular
    values to 1e-10 relative."""
    rng = np.random.default_rng(9)
    sv = clustered_spectrum(rng, 16, 16)
    m = len(sv)
    X = haar(rng, m) @ np.diag(sv) @ haar(rng, m).T
    s, U, VT = ctx.svd_dense(ctx._dev(X.copy()))
    s = s.cpu().numpy()
    sl = np.linalg.svd(X, compute_uv=False)
    big = sl > 1e-6 * sl[0]          # below that, FP64 storage of X alone perturbs by > 1e-10 relative
    assert np.max(np.abs(s - sl)[big] / sl[big]) < 1e-10


def test_dense_svd_cluster_subspaces(ctx):
    """Clusters of 16 values at relative spacing 1e-10 (the stress family):
    the twisted vectors alone collapse inside a cluster; after the cluster
    refinement every cluster's left and right subspaces match the exact ones
    to the gap-aware bar max(1e-8, 100 eps ||X|| / gap), vectors inside a
    cluster are orthonormal to 1e-13, and vectors of different clusters are
    orthogonal to the same gap-aware bar (independently computed vectors
    cannot be more orthogonal than their own accuracy)."""
    rng = np.random.default_rng(21)
    sv = clustered_spectrum(rng, 32, 16, lo=1e-6)
    m = len(sv)
    Ux, Vx = haar(rng, m), haar(rng, m)
    X = Ux @ np.diag(sv) @ Vx.T
    s, U, VT = ctx.svd_dense(ctx._dev(X.copy()))
    s, U, VT = s.cpu().numpy(), U.cpu().numpy(), VT.cpu().numpy()
    eps = np.finfo(float).eps
    cl = np.arange(m) // 16
    gap = np.abs(sv[:, None] - sv[None, :])
    same = cl[:, None] == cl[None, :]
    bound = np.where(same, 1e-13, np.maximum(1e-8, 100 * eps * sv[0] / np.where(same, 1.0, gap)))
    np.fill_diagonal(bound, 1e-13)
    assert np.all(np.abs(U.T @ U - np.eye(m)) <= bound)
    assert np.all(np.abs(VT @ VT.T - np.eye(m)) <= bound)
    for c in range(32):
        grp = list(range(16 * c, 16 * c + 16))
        lo = sv[grp[-1]] - (sv[grp[-1] + 1] if grp[-1] + 1 < m else 0.0)
        hi = (sv[grp[0] - 1] - sv[grp[0]]) if grp[0] > 0 else np.inf
        bar = max(1e-8, 100 * eps * sv[0] / min(lo, hi))
        assert subspace_angle(U[:, grp], Ux[:, grp]) < bar
        assert subspace_angle(VT[grp].T, Vx[:, grp]) < bar
