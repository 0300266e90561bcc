"""The CRT product fused with its reconstruction (crt_fused_kernel, csrc/crt.cu):
the products with the implicit Q of the exact-Gram mode keep every modulus's
accumulator on the SM and write FP64 directly.  It must equal the two-pass
product (residues of the product in HBM) + reconstruction bit for bit:
EXCALIBUR_B200_FUSED_APPLY=1 selects the fused path, =0 the two-pass path.
Both operand layouts are covered: the recomputed residues of X's columns
(K-major, bbt_exact_apply_q) and the Gram's kept residue planes read MN-major
(the pipeline's V back-transform, by crt_kernel or, with enough row blocks,
by crt_apply_kernel)."""
import os

import numpy as np
import pytest

import oracle
from gpu_util import context

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return context()


def with_env(value, fn):
    old = os.environ.get("EXCALIBUR_B200_FUSED_APPLY")
    try:
        if value is None:
            os.environ.pop("EXCALIBUR_B200_FUSED_APPLY", None)
        else:
            os.environ["EXCALIBUR_B200_FUSED_APPLY"] = value
        return fn()
    finally:
        if old is None:
            os.environ.pop("EXCALIBUR_B200_FUSED_APPLY", None)
        else:
            os.environ["EXCALIBUR_B200_FUSED_APPLY"] = old


# m sets the modulus count (17..19 for 53-bit rows times 80-bit columns);
# rows and k are not multiples of the 128 x 128 tile
@pytest.mark.parametrize("m,n,k", [(40, 3001, 40), (200, 20000, 333), (1000, 9000, 1000), (1500, 6000, 130)])
def test_fused_apply_equals_two_pass(ctx, m, n, k):
    rng = np.random.default_rng(m + k)
    X = rng.standard_normal((m, n)) * np.exp(rng.uniform(-3, 3, (m, 1)))
    Xd = ctx._dev(X)
    _, _, Rpt, sc = ctx.exact_local_qr(Xd)
    Z = ctx._dev(rng.standard_normal((k, m)))
    two = with_env("0", lambda: ctx.exact_apply_q(Xd, sc, Rpt, Z).cpu().numpy())
    one = with_env("1", lambda: ctx.exact_apply_q(Xd, sc, Rpt, Z).cpu().numpy())
    assert np.all(np.isfinite(one))
    assert np.array_equal(one, two)


# the second row set has more 128-row blocks than the B200 has SMs, so the
# two-pass product runs the kernel that keeps A's blocks in shared memory
@pytest.mark.parametrize("rows", [(5000, 3700), (20000, 19300)])
def test_fused_pipeline_back_transform_bitwise(ctx, rows):
    """The V back-transform from the kept residue planes (MN-major A operand)."""
    rng = np.random.default_rng(12)
    m, P, precision = 300, 2, 2
    blocks = [rng.standard_normal((m, n)) for n in rows]
    pub, priv = oracle.reference_seeds(3, P)

    def run():
        s, U, VT = ctx.fedsvd([ctx._dev(b.copy()) for b in blocks], pub, priv, precision=precision)
        return s.cpu().numpy(), U.cpu().numpy(), [v.cpu().numpy() for v in VT]

    s0, U0, V0 = with_env("0", run)
    s1, U1, V1 = with_env("1", run)
    assert np.array_equal(s0, s1) and np.array_equal(U0, U1)
    for a, b in zip(V0, V1):
        assert np.array_equal(a, b)
