"""The reference's random orthogonal matrix generators (bbtsvd.hpp:42-43,
Excalibur src/bbtsvd.cpp:301-331, 370-395) as exported by
libexcalibur_b200.so under their C++ signatures.  They are random-number
generation on the host through the LAPACK the process links (dlarnv,
dlarfg, dorgqr), the same calls in the same order as the reference: against
the reference's build over the same LAPACK the outputs and glibc's rand()
state afterwards are identical (gen__*.npz, written by
tests/golden/make_golden.py).  No GPU is needed."""
import ctypes as C
import glob
import os
import site

import numpy as np
import pytest

D = C.POINTER(C.c_double)


def _openblas():
    for d in site.getsitepackages():
        hits = glob.glob(os.path.join(d, "scipy.libs", "libscipy_openblas-*.so"))
        if hits:
            return hits[0]
    return None


@pytest.fixture(scope="module")
def lib():
    blas = _openblas()
    if blas is None:
        pytest.skip("no LAPACK library in this environment")
    C.CDLL(blas, mode=C.RTLD_GLOBAL)   # the process's LAPACK, found by the library at run time
    from excalibur_b200 import _lib
    if not os.path.exists(_lib.LIBPATH):
        pytest.skip("library not built")
    return C.CDLL(_lib.LIBPATH)


def p(a):
    return a.ctypes.data_as(D)


@pytest.mark.parametrize("name", ["house_row7", "house_col6"])
def test_random_orthogonal_house(lib, golden, name):
    g = golden(f"gen__{name}")
    m = int(g["m"])
    f = lib._Z33generate_random_orthogonal_matriximPdS_j
    f.restype = None
    f.argtypes = [C.c_int, C.c_size_t, D, D, C.c_uint]
    house, tau = np.zeros(m * m), np.zeros(max(m - 1, 1))
    f(int(g["layout"]), m, p(house), p(tau), int(g["seed"]))
    assert np.array_equal(house, g["house"]) and np.array_equal(tau, g["tau"])
    assert C.CDLL(None).rand() == int(g["rand_after"])


@pytest.mark.parametrize("name", ["orth_tall9x4", "orth_wide4x9"])
def test_random_orthogonal(lib, golden, name):
    g = golden(f"gen__{name}")
    m, n = int(g["m"]), int(g["n"])
    f = lib._Z33generate_random_orthogonal_matrixmmPdj
    f.restype = None
    f.argtypes = [C.c_size_t, C.c_size_t, D, C.c_uint]
    x = np.zeros(m * n)
    f(m, n, p(x), int(g["seed"]))
    assert np.array_equal(x, g["x"])
    q = x.reshape(m, n)
    gram = q.T @ q if m >= n else q @ q.T
    assert np.abs(gram - np.eye(min(m, n))).max() < 1e-14
    assert C.CDLL(None).rand() == int(g["rand_after"])
