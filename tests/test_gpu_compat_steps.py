"""The per-step helpers of the reference's bbtsvd.hpp (ldl_decomposition,
dstqds, dpqds, inverse_iteration, one_pair_singular_vector_twisted_
factorization, generate_house, mmap_drot; Excalibur src/bbtsvd.cpp:54-164,
970-978) as exported by libexcalibur_b200.so under the reference's own C++
signatures (called here by their mangled names, as a program linked against
the library would), against the reference's outputs (step__*.npz, written
by tests/golden/make_golden.py from the reference's build).  The recurrences
run on the GPU in the reference's order of operations: bit-exact; vectors
normalised by a 2-norm agree to rounding (the reference's BLAS dnrm2)."""
import ctypes as C

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu
D = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def lib():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from excalibur_b200 import _lib
    return _lib.load()


def p(a):
    return a.ctypes.data_as(D)


def fn(L, name, args):
    f = getattr(L, name)
    f.restype = None
    f.argtypes = args
    return f


@pytest.mark.parametrize("name", sorted(cases.step_cases()))
def test_step_helpers_match_reference(lib, golden, name):
    g = golden(f"step__{name}")
    a, b = g["alpha"].copy(), g["beta"].copy()
    n = len(a)
    bb = b.copy() if n > 1 else np.zeros(1)
    i, dbl = C.c_int, C.c_double
    ldl = fn(lib, "_Z17ldl_decompositioniPdS_S_S_", [i, D, D, D, D])
    l, d = np.zeros(max(n - 1, 1)), np.zeros(n)
    ldl(n, p(a), p(bb), p(l), p(d))
    assert np.array_equal(l[:n - 1], g["l"]) and np.array_equal(d, g["d"])
    tau = float(g["omega"]) ** 2
    dst = fn(lib, "_Z6dstqdsiPdS_dS_S_S_", [i, D, D, dbl, D, D, D])
    lp, dp, s = np.zeros(max(n - 1, 1)), np.zeros(n), np.zeros(n)
    dst(n, p(l), p(d), tau, p(lp), p(dp), p(s))
    assert np.array_equal(lp[:n - 1], g["lp"]) and np.array_equal(dp, g["dp"]) and np.array_equal(s, g["s"])
    dpq = fn(lib, "_Z5dpqdsiPdS_dS_S_S_", [i, D, D, dbl, D, D, D])
    up, rp, pp = np.zeros(max(n - 1, 1)), np.zeros(n), np.zeros(n)
    dpq(n, p(l), p(d), tau, p(up), p(rp), p(pp))
    assert np.array_equal(up[:n - 1], g["up"]) and np.array_equal(rp, g["rp"]) and np.array_equal(pp, g["p"])
    inv = fn(lib, "_Z17inverse_iterationiiPdS_S_i", [i, i, D, D, D, i])
    vi = np.zeros(2 * n)
    inv(n, int(g["twist"]), p(lp), p(up), p(vi), 2)
    assert np.max(np.abs(vi - g["vi"])) < 1e-15
    one = fn(lib, "_Z46one_pair_singular_vector_twisted_factorizationiidPdS_S_S_S_S_",
             [i, i, dbl, D, D, D, D, D, D])
    v, u = np.zeros(n), np.zeros(n * 3)
    one(n, 3, float(g["omega"]), p(l), p(d), p(a), p(bb), p(v), p(u))
    assert np.max(np.abs(v - g["v"])) < 1e-15 and np.max(np.abs(u - g["u"])) < 1e-15
    house = fn(lib, "_Z14generate_houseiPdiS_", [i, D, i, D])
    hx = g["house_in"].copy()
    inc = int(g["house_inc"])
    beta = np.zeros(1)
    house(len(hx) // inc, p(hx), inc, p(beta))
    assert np.array_equal(hx, g["house_out"]) and np.array_equal(beta, g["house_beta"])
    rot = fn(lib, "_Z9mmap_drotmPdmS_mdd", [C.c_size_t, D, C.c_size_t, D, C.c_size_t, dbl, dbl])
    x, y = a.copy(), np.resize(b, n).copy()
    rot(n, p(x), 1, p(y), 1, float(g["drot_c"]), float(g["drot_s"]))
    assert np.array_equal(x, g["drot_x"]) and np.array_equal(y, g["drot_y"])


@pytest.mark.parametrize("name", ["shuffle_left7x5", "unshuffle_left7x5", "shuffle_right6x9",
                                  "unshuffle_right6x9", "shuffle_left8x3"])
def test_shuffle_matrix(lib, golden, name):
    """shuffle_matrix (bbtsvd.cpp:398-427): the permutation drawn on the host
    with the reference's calls, the row or column swaps on the GPU; the
    result and glibc's rand() state afterwards are the reference's."""
    g = golden(f"gen__{name}")
    m, n = int(g["m"]), int(g["n"])
    x = g["x_in"].copy()
    f = fn(lib, "_Z14shuffle_matrixmmPdjbb", [C.c_size_t, C.c_size_t, D, C.c_uint, C.c_bool, C.c_bool])
    f(m, n, p(x), int(g["seed"]), bool(g["is_left"]), bool(g["unshuffle"]))
    assert np.array_equal(x, g["x_out"])
    libc = C.CDLL(None)
    assert libc.rand() == int(g["rand_after"])
