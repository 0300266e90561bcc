"""Split-precision path (precision mode 1): the tcgen05 BF16x3 sketch
product, the sketch-preconditioned Cholesky-QR local QR with its FP64
refinement pass, and the whole pipeline with precision=1 against the
reference's own outputs (golden) and LAPACK."""
import numpy as np
import pytest

import cases
import oracle
from gpu_util import context, gap_groups, subspace_angle
from oracle import pipeline

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return context()


def signs(S, n):
    """The +-1 entries of the bf16 sketch (bit patterns 0x3F80 / 0xBF80)."""
    b = S.cpu().numpy()[:, :n].astype(np.int64) & 0xFFFF
    assert np.all((b == 0x3F80) | (b == 0xBF80))
    return np.where(b == 0x3F80, 1.0, -1.0)


@pytest.mark.parametrize("m,n,N", [(200, 5003, 512), (100, 1000, 256), (130, 64, 128), (7, 20000, 128),
                                   (300, 70001, 640)])
def test_sketch_bf16x3(ctx, m, n, N):
    """Y = X S^T on the tensor cores against the FP64 product: the error per
    entry, relative to its row's scale sqrt(n) rms(x_i), stays at FP32
    accumulation level (a single bf16 piece would leave ~1e-3)."""
    rng = np.random.default_rng(m * 7 + n)
    X = rng.standard_normal((m, n)) * np.exp(rng.uniform(-3.0, 3.0, (m, 1)))
    S = ctx.rademacher(N, n, 11 + m)
    Sd = signs(S, n)
    assert abs(Sd.mean()) < 0.05
    Y = ctx.sketch_bf16x3(ctx._dev(X), S, N).cpu().numpy()
    ref = X @ Sd.T
    scale = np.sqrt(n) * np.sqrt(np.mean(X ** 2, axis=1, keepdims=True))
    err = np.abs(Y - ref) / scale
    assert err.max() < 1e-5, err.max()


def orthonormal(rng, rows, cols):
    q, r = np.linalg.qr(rng.standard_normal((rows, cols)))
    return q * np.sign(np.diag(r))


@pytest.mark.parametrize("m,n,cond", [(100, 20000, 1e6), (64, 3000, 1e3), (200, 6000, 1e6), (33, 4001, 1e2)])
def test_mixed_local_qr(ctx, m, n, cond):
    """A = X^T = Q R with Q = Q_p W orthonormal to 1e-13, the residual at
    FP64 level, R equal to LAPACK dgeqrf's R -- row signs included, recovered
    from the top block of Q -- to cond * eps, and the singular values of R
    those of X."""
    rng = np.random.default_rng(m + n)
    sv = np.geomspace(1.0, 1.0 / cond, m)
    X = (orthonormal(rng, m, m) * sv) @ orthonormal(rng, n, m).T
    Xd = ctx._dev(X.copy())
    Rt, Wt = ctx.mixed_local_qr(Xd)
    R, W = Rt.cpu().numpy().T, Wt.cpu().numpy().T
    Qp = Xd.cpu().numpy().T
    assert np.all(np.tril(R, -1) == 0.0)
    Q = Qp @ W
    assert np.max(np.abs(Q.T @ Q - np.eye(m))) < 1e-13
    assert np.linalg.norm(X.T - Q @ R) / np.linalg.norm(X) < 1e-14
    Rl = np.linalg.qr(X.T, mode="r")   # dgeqrf
    assert np.all(np.sign(np.diag(R)) == np.sign(np.diag(Rl)))
    assert np.max(np.abs(R - Rl)) / np.max(np.abs(Rl)) < 1e-15 * cond * 100
    sl = np.linalg.svd(Rl, compute_uv=False)
    sr = np.linalg.svd(R, compute_uv=False)
    assert np.max(np.abs(sr - sl) / sl) < 1e-15 * cond * 10


def run(ctx, blocks, seed, precision, top_k=-1, svd_mode=1):
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    dev = [ctx._dev(b.copy()) for b in blocks]
    s, U, VT = ctx.fedsvd(dev, pub, priv, top_k=top_k, svd_mode=svd_mode, precision=precision)
    return (s.cpu().numpy(), None if U is None else U.cpu().numpy(),
            None if VT is None else [v.cpu().numpy() for v in VT])


@pytest.mark.parametrize("precision", [1, 2])
@pytest.mark.parametrize("name", sorted(cases.pipeline_cases()))
def test_mixed_pipeline_matches_reference(ctx, golden, name, precision):
    """precision 1 (sketch + Cholesky QR) and 2 (sketch + exact Gram)
    reproduce the reference's outputs on its own inputs: singular values to
    1e-12 relative, U and every FinalVT_c to 1e-9 (dgeqrf's row signs are
    recovered, so the vectors match, not only their subspaces)."""
    g = golden(f"pipe__{name}")
    blocks, seed = cases.pipeline_cases()[name]
    s, U, VT = run(ctx, blocks, seed, precision)
    assert len(s) == len(g["sigma"])
    assert np.max(np.abs(s - g["sigma"]) / g["sigma"]) < 1e-12
    assert np.max(np.abs(U - g["U"])) < 1e-9
    for c, v in enumerate(VT):
        assert np.max(np.abs(v - g[f"VT{c}"])) < 1e-9


@pytest.mark.parametrize("precision", [1, 2])
@pytest.mark.parametrize("name", sorted(cases.pipeline_mode_cases()))
def test_mixed_pipeline_modes(ctx, golden, name, precision):
    g = golden(f"pipe__{name}")
    case, mode, topk = cases.pipeline_mode_cases()[name]
    blocks, seed = cases.pipeline_cases()[case]
    s, U, VT = run(ctx, blocks, seed, precision, top_k=topk, svd_mode=mode)
    assert np.max(np.abs(s - g["sigma"]) / g["sigma"]) < 1e-12
    if mode != 3:
        assert np.max(np.abs(U - g["U"])) < 1e-9
    if mode != 2:
        for c, v in enumerate(VT):
            assert np.max(np.abs(v - g[f"VT{c}"])) < 1e-9


@pytest.mark.parametrize("precision", [1, 2])
def test_mixed_vs_plain_geometric(ctx, precision):
    """The tall-skinny family (s from 1 to 1e-6, Haar factors) at reduced
    rows: mixed and plain agree with the exact spectrum to the conditioning
    bound, with each other to 1e-10 relative on sigma >= 1e-4, and the
    well-posed left subspaces agree to 1e-8."""
    rng = np.random.default_rng(12)
    m, n, P = 200, 12000, 2
    Uq = orthonormal(rng, P * n, m)
    Vq = orthonormal(rng, m, m)
    sv = np.geomspace(1.0, 1e-6, m)
    Xt = (Uq * sv) @ Vq.T
    blocks = [Xt[c * n:(c + 1) * n].T.copy() for c in range(P)]
    s0, U0, V0 = run(ctx, blocks, 3, 0)
    s1, U1, V1 = run(ctx, blocks, 3, precision)
    assert np.max(np.abs(s1 - sv) / sv) < 1e-10 * 1e4
    big = sv >= 1e-4
    assert np.max(np.abs(s1 - s0)[big] / s0[big]) < 1e-10
    X = np.concatenate(blocks, axis=1)
    assert np.max(np.abs(U1 @ np.diag(s1) @ np.concatenate(V1, axis=1) - X)) < 1e-13
    for grp in gap_groups(s0, 1e-3):
        if s0[grp[-1]] < 1e-4:
            continue
        assert subspace_angle(U1[:, grp], U0[:, grp]) < 1e-8


@pytest.mark.parametrize("precision", [1, 2])
def test_mixed_batched_graph_and_tune(ctx, precision):
    """Uneven participants on concurrent streams in both split-precision
    modes: eager, captured and replayed calls all match the oracle."""
    rng = np.random.default_rng(35)
    m = 32
    rows = [int(r) for r in rng.integers(200, 900, 10)]
    blocks = [rng.standard_normal((m, n)) * 10.0 ** rng.uniform(-2, 2) for n in rows]
    st, nb, ms = ctx.fedsvd_tune(m, rows, precision=precision)
    assert st in (1, 4, 8, 16) and ms > 0
    pub, priv = oracle.reference_seeds(4, len(blocks))
    so, Uo, VTo = pipeline.run(blocks, pub, priv)
    dev = [ctx._dev(b.copy()) for b in blocks]
    for call in range(3):
        for d, b in zip(dev, blocks):
            d.copy_(ctx.torch.as_tensor(b, device=d.device))
        s, U, VT = ctx.fedsvd(dev, pub, priv, precision=precision)
        s, U = s.cpu().numpy(), U.cpu().numpy()
        assert np.max(np.abs(s - so) / so) < 1e-12, call
        assert np.max(np.abs(U - Uo)) < 1e-9, call
        for v, w in zip(VT, VTo):
            assert np.max(np.abs(v.cpu().numpy() - w)) < 1e-9, call
