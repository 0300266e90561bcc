"""DecentralizedClient::run() on one GPU (P participants as device buffers)
against the reference's own pipeline outputs (golden), the oracle pipeline
and the LAPACK FP64 SVD."""
import numpy as np
import pytest

import cases
import oracle
from gpu_util import context, gap_groups, subspace_angle
from oracle import pipeline

pytestmark = pytest.mark.gpu
PIPES = sorted(cases.pipeline_cases())


@pytest.fixture(scope="module")
def ctx():
    return context()


def run(ctx, blocks, seed, top_k=-1, svd_mode=1):
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    dev = [ctx._dev(b.copy()) for b in blocks]
    s, U, VT = ctx.fedsvd(dev, pub, priv, top_k=top_k, svd_mode=svd_mode)
    return (s.cpu().numpy(), None if U is None else U.cpu().numpy(),
            None if VT is None else [v.cpu().numpy() for v in VT])


@pytest.mark.parametrize("name", sorted(cases.pipeline_mode_cases()))
def test_pipeline_modes_match_reference(ctx, golden, name):
    """svd_mode 0 (the reference's dbdsdc on the leading k x k bidiagonal),
    2 (left only), 3 (right only) and top-k (client.cpp:186-192, 971-985)."""
    g = golden(f"pipe__{name}")
    case, mode, topk = cases.pipeline_mode_cases()[name]
    blocks, seed = cases.pipeline_cases()[case]
    s, U, VT = run(ctx, blocks, seed, top_k=topk, svd_mode=mode)
    assert len(s) == len(g["sigma"])
    assert np.max(np.abs(s - g["sigma"]) / g["sigma"]) < 1e-12
    if mode != 3:
        assert np.max(np.abs(U - g["U"])) < 1e-9
    else:
        assert U is None
    if mode != 2:
        for c, v in enumerate(VT):
            assert np.max(np.abs(v - g[f"VT{c}"])) < 1e-9
    else:
        assert VT is None


@pytest.mark.parametrize("name", PIPES)
def test_pipeline_matches_reference(ctx, golden, name):
    g = golden(f"pipe__{name}")
    blocks, seed = cases.pipeline_cases()[name]
    s, U, VT = run(ctx, blocks, seed)
    assert len(s) == len(g["sigma"])
    assert np.max(np.abs(s - g["sigma"]) / g["sigma"]) < 1e-12
    assert np.max(np.abs(U - g["U"])) < 1e-9
    for c, v in enumerate(VT):
        assert np.max(np.abs(v - g[f"VT{c}"])) < 1e-9


@pytest.mark.parametrize("name", PIPES)
def test_pipeline_matches_oracle_and_lapack(ctx, name):
    blocks, seed = cases.pipeline_cases()[name]
    s, U, VT = run(ctx, blocks, seed)
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    so, Uo, VTo = pipeline.run(blocks, pub, priv)
    assert np.max(np.abs(s - so) / so) < 1e-12
    assert np.max(np.abs(U - Uo)) < 1e-9
    X = np.concatenate(blocks, axis=1)
    Ul, sl, Vl = np.linalg.svd(X, full_matrices=False)
    assert np.max(np.abs(s - sl) / sl) < 1e-10
    V = np.concatenate(VT, axis=1).T
    for grp in gap_groups(sl):
        assert subspace_angle(U[:, grp], Ul[:, grp]) < 1e-8
        assert subspace_angle(V[:, grp], Vl[grp].T) < 1e-8


def test_pipeline_host_entry_equals_device_entry(ctx):
    blocks, seed = cases.pipeline_cases()["p3_uneven"]
    s, U, VT = run(ctx, blocks, seed)
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    s2, U2, VT2 = ctx.fedsvd_host(blocks, pub, priv)
    assert np.array_equal(s, s2)
    assert np.array_equal(U, U2)
    for a, b in zip(VT, VT2):
        assert np.array_equal(a, b)


def test_pipeline_geometric_spectrum(ctx):
    """The c2 family at reduced rows: X = U diag(s) V^T, s from 1 to 1e-6."""
    rng = np.random.default_rng(11)
    m, n, P = 200, 6000, 2
    Uq, _ = np.linalg.qr(rng.standard_normal((P * n, m)))
    Vq, _ = np.linalg.qr(rng.standard_normal((m, m)))
    sv = np.geomspace(1.0, 1e-6, m)
    Xt = (Uq * sv) @ Vq.T                    # row-stacked (P*n) x m
    blocks = [Xt[c * n:(c + 1) * n].T.copy() for c in range(P)]
    s, U, VT = run(ctx, blocks, 3)
    assert np.max(np.abs(s - sv) / sv) < 1e-10 * 1e4   # conditioning bound for s_min ~ 1e-6
    X = np.concatenate(blocks, axis=1)
    assert np.max(np.abs(U @ np.diag(s) @ np.concatenate(VT, axis=1) - X)) < 1e-13


def test_batched_local_qr_graph_replay(ctx):
    """Ten participants (c3-like uneven rows): the local QRs run on
    concurrent streams, eagerly on the first call, captured into a CUDA graph
    on the second and replayed on the third; every call matches the oracle."""
    rng = np.random.default_rng(33)
    m = 32
    rows = [int(r) for r in rng.integers(200, 900, 10)]
    blocks = [rng.standard_normal((m, n)) * 10.0 ** rng.uniform(-2, 2) for n in rows]
    pub, priv = oracle.reference_seeds(4, len(blocks))
    so, Uo, VTo = pipeline.run(blocks, pub, priv)
    dev = [ctx._dev(b.copy()) for b in blocks]
    for call in range(3):
        for d, b in zip(dev, blocks):
            d.copy_(ctx.torch.as_tensor(b, device=d.device))
        s, U, VT = ctx.fedsvd(dev, pub, priv)
        s, U = s.cpu().numpy(), U.cpu().numpy()
        assert np.max(np.abs(s - so) / so) < 1e-12, call
        assert np.max(np.abs(U - Uo)) < 1e-9, call
        for v, w in zip(VT, VTo):
            assert np.max(np.abs(v.cpu().numpy() - w)) < 1e-9, call


def test_autotuned_batched_local_qr(ctx):
    rng = np.random.default_rng(34)
    m = 24
    rows = [int(r) for r in rng.integers(150, 600, 9)]
    blocks = [rng.standard_normal((m, n)) for n in rows]
    st, nb, ms = ctx.fedsvd_tune(m, rows)
    assert st in (1, 4, 8, 16) and nb in (64, 128) and ms > 0
    pub, priv = oracle.reference_seeds(6, len(blocks))
    so, Uo, VTo = pipeline.run(blocks, pub, priv)
    s, U, VT = ctx.fedsvd([ctx._dev(b.copy()) for b in blocks], pub, priv)
    assert np.max(np.abs(s.cpu().numpy() - so) / so) < 1e-12
    assert np.max(np.abs(U.cpu().numpy() - Uo)) < 1e-9


def _clustered_blocks(rng, m, n, P, clusters, size, gap=1e-10, lo=1e-3):
    """X = Ux diag(s) Vx^T (m x P n) with `clusters` clusters of `size` values
    at relative spacing `gap`, centres log-uniform in [lo, 1]; blocks X_c."""
    c = np.exp(rng.uniform(np.log(lo), 0.0, clusters))
    sv = np.sort(np.concatenate([ci * (1.0 + gap * np.arange(size)) for ci in c]))[::-1]
    sv = np.concatenate([sv, np.geomspace(lo / 2, lo / 4, m - len(sv))]) if len(sv) < m else sv
    Ux, _ = np.linalg.qr(rng.standard_normal((m, m)))
    Vx, _ = np.linalg.qr(rng.standard_normal((P * n, m)))
    X = (Ux * sv) @ Vx.T
    return [X[:, c * n:(c + 1) * n].copy() for c in range(P)], sv


@pytest.mark.parametrize("top_k", [-1, 40])
def test_pipeline_mode0_clustered_orthogonal(ctx, top_k):
    """svd_mode 0 stands in for the reference's dbdsdc (client.cpp:975-980),
    which keeps singular vectors orthogonal inside tight clusters.  Clusters
    of 16 values at relative spacing 1e-10: the vectors of every cluster are
    orthonormal to 1e-12 (the twisted vectors alone collapse onto each
    other), and each cluster's left and right subspaces match LAPACK's to the
    gap-aware bar max(1e-8, 100 eps ||X|| / gap)."""
    rng = np.random.default_rng(77)
    m, n, P = 96, 700, 2
    blocks, sv = _clustered_blocks(rng, m, n, P, clusters=5, size=16)
    s, U, VT = run(ctx, blocks, 8, top_k=top_k, svd_mode=0)
    X = np.concatenate(blocks, axis=1)
    Ul, sl, Vl = np.linalg.svd(X, full_matrices=False)
    k = len(s)
    assert k == (m if top_k < 0 else top_k)
    V = np.concatenate(VT, axis=1).T
    assert np.all(np.isfinite(U[:, :k])) and np.all(np.isfinite(V[:, :k]))
    # with top_k the reference's dbdsdc factors the LEADING k x k bidiagonal
    # (client.cpp:975-980): its values are not X's top k (the golden mode-0
    # top-k case pins that); the clusters of its spectrum are checked for
    # orthogonality, the full SVD against LAPACK as well
    ref = sl if top_k < 0 else s
    if top_k < 0:
        assert np.max(np.abs(s - sl)) < 1e-12 * sl[0]
    eps = np.finfo(float).eps
    clusters = 0
    for g in gap_groups(ref[:k], rel_gap=1e-7):
        if len(g) < 2:
            continue
        clusters += 1
        assert np.max(np.abs(U[:, g].T @ U[:, g] - np.eye(len(g)))) < 1e-12
        assert np.max(np.abs(V[:, g].T @ V[:, g] - np.eye(len(g)))) < 1e-12
        if top_k < 0:
            lo_gap = sl[g[-1]] - sl[g[-1] + 1] if g[-1] + 1 < len(sl) else sl[g[-1]]
            hi_gap = sl[g[0] - 1] - sl[g[0]] if g[0] > 0 else np.inf
            bar = max(1e-8, 100 * eps * sl[0] / min(lo_gap, hi_gap))
            assert subspace_angle(U[:, g], Ul[:, g]) < bar
            assert subspace_angle(V[:, g], Vl[g].T) < bar
    assert clusters >= (5 if top_k < 0 else 0)
