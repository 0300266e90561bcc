"""The masks of the reference's bbtsvd.hpp off the opt_control 1/3 path
(naive_givens_mask_parallel, givens_mask_cache_optimized_parallel,
block_mask, shuffle_block_mask, house_mask, householder_reflector_mask;
Excalibur src/bbtsvd.cpp:190-299, 429-531, 670-726) as exported by
libexcalibur_b200.so under their C++ signatures, called by their mangled
names.  Against the reference's build (omask__*.npz, written by
tests/golden/make_golden.py): the rotation masks to the last bit (the
tables are drawn with the reference's calls, each product and sum rounded
on its own) or to rounding where the reference rotates with BLAS drot; the
Householder masks to rounding (Q formed and multiplied on the GPU where the
reference calls dormqr); glibc's rand() state afterwards exactly.  Blocks of
the full block size, whose last reflector the reference reads from one past
its tau array, are checked against Q built here from the exported
generator, and by masking then unmasking."""
import ctypes as C
import glob
import os
import site

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu
D = C.POINTER(C.c_double)
SZ, B, U = C.c_size_t, C.c_bool, C.c_uint

NAMES = {
    "naive": ("_Z26naive_givens_mask_parallelmmmPdbbj", [SZ, SZ, SZ, D, B, B, U]),
    "cached": ("_Z36givens_mask_cache_optimized_parallelmmmPdbbj", [SZ, SZ, SZ, D, B, B, U]),
    "block": ("_Z10block_maskmmmPdbbj", [SZ, SZ, SZ, D, B, B, U]),
    "shufblock": ("_Z18shuffle_block_maskmmmiPdbbj", [SZ, SZ, SZ, C.c_int, D, B, B, U]),
    "house": ("_Z10house_maskmmmPdbbj", [SZ, SZ, SZ, D, B, B, U]),
    "reflector": ("_Z26householder_reflector_maskmmmPdbbj", [SZ, SZ, SZ, D, B, B, U]),
}


@pytest.fixture(scope="module")
def lib():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    hits = [h for d in site.getsitepackages() for h in glob.glob(os.path.join(d, "scipy.libs", "libscipy_openblas-*.so"))]
    if not hits:
        pytest.skip("no LAPACK library in this environment")
    C.CDLL(hits[0], mode=C.RTLD_GLOBAL)   # the process's LAPACK, found by the library at run time
    from excalibur_b200 import _lib
    return _lib.load()


def p(a):
    return a.ctypes.data_as(D)


def fn(L, key):
    name, args = NAMES[key]
    f = getattr(L, name)
    f.restype = None
    f.argtypes = args
    return f


def call(L, key, m, n, size, rounds, x, mask, left, seed):
    if key == "shufblock":
        fn(L, key)(m, n, size, rounds, p(x), bool(mask), bool(left), seed)
    else:
        fn(L, key)(m, n, size, p(x), bool(mask), bool(left), seed)


@pytest.mark.parametrize("name", sorted(cases.OTHER_MASK_CASES))
def test_mask_matches_reference(lib, golden, name):
    key, m, n, size, rounds, mask, left, seed = cases.OTHER_MASK_CASES[name]
    g = golden(f"omask__{name}")
    x = g["x_in"].copy()
    call(lib, key, m, n, size, rounds, x, mask, left, seed)
    scale = np.abs(g["x_out"]).max()
    if key == "cached":
        assert np.array_equal(x, g["x_out"])
    elif key == "naive":
        assert np.abs(x - g["x_out"]).max() <= 1e-14 * scale
    else:
        assert np.abs(x - g["x_out"]).max() <= 1e-12 * scale
    assert C.CDLL(None).rand() == int(g["rand_after"])


def block_q(lib, rb, seed):
    """Q = H_0 ... H_{rb-2} of generate_random_orthogonal_matrix(row-major,
    rb, seed) (the library's host generator, pinned by gen__house_row7)."""
    f = lib._Z33generate_random_orthogonal_matriximPdS_j
    f.restype = None
    f.argtypes = [C.c_int, C.c_size_t, D, D, C.c_uint]
    house, tau = np.zeros(rb * rb), np.zeros(max(rb - 1, 1))
    f(101, rb, p(house), p(tau), seed)
    V = house.reshape(rb, rb)
    Q = np.eye(rb)
    for j in range(rb - 2, -1, -1):
        v = np.zeros(rb)
        v[j] = 1.0
        v[j + 1:] = V[j + 1:, j]
        Q -= tau[j] * np.outer(v, v @ Q)
    return Q


@pytest.mark.parametrize("m,n,bs,left,mask", [(7, 5, 3, 1, 1), (6, 9, 4, 0, 0), (10, 4, 5, 1, 0), (3, 11, 2, 0, 1)])
def test_block_mask_full_blocks(lib, m, n, bs, left, mask):
    rng = np.random.default_rng(m * n + bs)
    x0 = rng.standard_normal((m, n))
    seed = 31 + bs
    k = m if left else n
    ref = x0.copy()
    for i in range(0, k, bs):
        rb = min(bs, k - i)
        Q = block_q(lib, rb, seed)
        op = Q if mask else Q.T
        if left:
            ref[i:i + rb, :] = op @ ref[i:i + rb, :]
        else:
            ref[:, i:i + rb] = ref[:, i:i + rb] @ op
    want = C.CDLL(None).rand()
    x = np.ascontiguousarray(x0.copy())
    call(lib, "block", m, n, bs, 0, x.reshape(-1), mask, left, seed)
    assert np.abs(x - ref).max() <= 1e-12 * np.abs(ref).max()
    assert C.CDLL(None).rand() == want


@pytest.mark.parametrize("key,m,n,size,rounds,left", [("block", 9, 7, 3, 0, 1), ("shufblock", 8, 10, 3, 3, 0),
                                                      ("shufblock", 9, 6, 4, 2, 1), ("cached", 9, 7, 5, 0, 0),
                                                      ("house", 8, 6, 5, 0, 1), ("reflector", 5, 9, 4, 0, 0)])
def test_mask_then_unmask(lib, key, m, n, size, rounds, left):
    rng = np.random.default_rng(m + 10 * n + size)
    x0 = rng.standard_normal(m * n)
    x = x0.copy()
    call(lib, key, m, n, size, rounds, x, 1, left, 77)
    assert np.abs(x - x0).max() > 1e-3
    call(lib, key, m, n, size, rounds, x, 0, left, 77)
    assert np.abs(x - x0).max() <= 1e-12 * np.abs(x0).max()
