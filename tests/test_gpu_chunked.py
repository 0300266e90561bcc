"""Passes over the long dimension in bounded chunks.

A participant's block can be far larger than the scratch a pass over it may
take (4 participants x 2000 x 10^6 FP64 in the largest workload), so the
sketch's bf16 pieces, the exact Gram's residue planes, the products with the
implicit Q and the long Ozaki products are formed in chunks whose size is
capped (EXCALIBUR_B200_CHUNK_BYTES overrides the cap).  Here the cap is set to
1-4 MiB so that a 100,000-column block runs in many chunks, and every result
is compared with the same call without chunking: the sketch and the Gram are
sums over the long dimension (chunks add partial sums), the products with Q
are independent per row."""
import os

import numpy as np
import pytest

import oracle
from gpu_util import context

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return context()


def _blocks(rng, m, n, P):
    Uq, _ = np.linalg.qr(rng.standard_normal((P * n, m)))
    Vq, _ = np.linalg.qr(rng.standard_normal((m, m)))
    sv = np.geomspace(1.0, 1e-4, m)
    Xt = (Uq * sv) @ Vq.T
    return [Xt[c * n:(c + 1) * n].T.copy() for c in range(P)]


def _run(ctx, blocks, precision, cap):
    pub, priv = oracle.reference_seeds(5, len(blocks))
    old = os.environ.get("EXCALIBUR_B200_CHUNK_BYTES")
    try:
        if cap:
            os.environ["EXCALIBUR_B200_CHUNK_BYTES"] = str(cap)
        else:
            os.environ.pop("EXCALIBUR_B200_CHUNK_BYTES", None)
        s, U, VT = ctx.fedsvd([ctx._dev(b.copy()) for b in blocks], pub, priv, precision=precision)
    finally:
        if old is None:
            os.environ.pop("EXCALIBUR_B200_CHUNK_BYTES", None)
        else:
            os.environ["EXCALIBUR_B200_CHUNK_BYTES"] = old
    return s.cpu().numpy(), U.cpu().numpy(), [v.cpu().numpy() for v in VT]


@pytest.mark.parametrize("precision", [1, 2])
@pytest.mark.parametrize("cap", [1 << 20, 4 << 20])
def test_chunked_long_dimension_equals_one_pass(ctx, precision, cap):
    rng = np.random.default_rng(40 + precision)
    m, n, P = 64, 100_000, 2
    blocks = _blocks(rng, m, n, P)
    s0, U0, VT0 = _run(ctx, blocks, precision, None)
    s1, U1, VT1 = _run(ctx, blocks, precision, cap)
    assert np.max(np.abs(s1 - s0) / s0) < 1e-12
    assert np.max(np.abs(U1 - U0)) < 1e-9
    for a, b in zip(VT1, VT0):
        assert np.max(np.abs(a - b)) < 1e-9
    X = np.concatenate(blocks, axis=1)
    sl = np.linalg.svd(X, compute_uv=False)
    assert np.max(np.abs(s1 - sl) / sl) < 1e-10


def test_chunked_exact_gram_is_exact(ctx):
    """The Gram of the 53-bit rows is an exact integer product: formed in
    K-chunks whose K-splits are summed by one reconstruction, it is the same
    double-double bit for bit."""
    rng = np.random.default_rng(3)
    X = rng.standard_normal((96, 120_000))
    old = os.environ.get("EXCALIBUR_B200_CHUNK_BYTES")
    try:
        os.environ.pop("EXCALIBUR_B200_CHUNK_BYTES", None)
        h0, l0 = (t.cpu().numpy() for t in ctx.gram_dd(ctx._dev(X)))
        os.environ["EXCALIBUR_B200_CHUNK_BYTES"] = str(1 << 20)
        h1, l1 = (t.cpu().numpy() for t in ctx.gram_dd(ctx._dev(X)))
    finally:
        if old is None:
            os.environ.pop("EXCALIBUR_B200_CHUNK_BYTES", None)
        else:
            os.environ["EXCALIBUR_B200_CHUNK_BYTES"] = old
    iu = np.triu_indices(96)
    assert np.array_equal(h1[iu], h0[iu]) and np.array_equal(l1[iu], l0[iu])
