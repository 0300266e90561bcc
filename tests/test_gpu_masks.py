"""Givens / block-shift data masks on the GPU, bit-exact against the
reference's golden outputs (bbtsvd.cpp:533-876)."""
import numpy as np
import pytest

import cases
import oracle
from gpu_util import context

pytestmark = pytest.mark.gpu
NAMES = sorted(cases.mask_cases())


@pytest.fixture(scope="module")
def ctx():
    return context()


@pytest.mark.parametrize("name", NAMES)
def test_mask_bit_exact(ctx, golden, name):
    g = golden(f"mask__{name}")
    x, passes, mask, is_left, seed, fn = cases.mask_cases()[name]
    t = ctx._dev(x.copy())
    f = ctx.givens_mask_cache_optimized_parallel_with_simd if fn == "givens" else ctx.block_shift_mask
    f(t, passes, mask, is_left, seed)
    assert np.array_equal(t.cpu().numpy(), g["y"])


@pytest.mark.parametrize("shape,is_left", [((1000, 1000), 1), ((1000, 1000), 0), ((2000, 777), 1),
                                           ((513, 4097), 0), ((8192, 64), 1)])
def test_mask_roundtrip_and_oracle(ctx, shape, is_left):
    rng = np.random.default_rng(sum(shape))
    x = rng.standard_normal(shape)
    t = ctx._dev(x.copy())
    ctx.block_shift_mask(t, 32, True, is_left, 1234)
    y = t.cpu().numpy()
    assert np.array_equal(y, oracle.block_shift_mask(x, 32, True, is_left, 1234))
    ctx.block_shift_mask(t, 32, False, is_left, 1234)
    assert np.max(np.abs(t.cpu().numpy() - x)) < 1e-13


def test_mask_leaves_rand_state_like_reference(ctx):
    import ctypes
    libc = ctypes.CDLL("libc.so.6")
    x = np.random.default_rng(0).standard_normal((33, 5))
    ctx.block_shift_mask(ctx._dev(x.copy()), 32, True, True, 77)
    a = libc.rand()
    oracle.block_shift_mask(x, 32, True, True, 77)
    b = oracle.lib().orc_rand()
    assert a == b
