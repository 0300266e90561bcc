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


def run(ctx, blocks, seed):
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    dev = [ctx._dev(b.copy()) for b in blocks]
    s, U, VT = ctx.fedsvd(dev, pub, priv)
    return s.cpu().numpy(), U.cpu().numpy(), [v.cpu().numpy() for v in VT]


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
