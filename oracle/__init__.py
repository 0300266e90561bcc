"""ORACLE — test infrastructure, not product code.

CPU restatement of the Excalibur hot path used to check the CUDA path.
Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs may import this package; the product (excalibur_b200) never does.

* ``liboracle.so`` (oracle/bbt_oracle.cpp): Sturm counts, bisection, twisted
  factorisation and the Givens data masks of Excalibur ``src/bbtsvd.cpp``,
  restated operation by operation.  Pinned bit-exactly (singular values,
  masks) against the reference's own sources compiled by ``make -C oracle
  ref`` — see tests/test_oracle_golden.py and tests/golden/.
* ``pipeline.py``: numpy restatement of ``DecentralizedClient::run()``
  (Excalibur ``src/client.cpp:447-1200``) for P participants held in one
  process, the ring all-reduce being a fixed-order sum.
"""
import ctypes as _C
import os as _os
import subprocess as _sp

import numpy as _np

_HERE = _os.path.dirname(_os.path.abspath(__file__))
_LIB = _os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build():
    """Compile liboracle.so (g++, seconds)."""
    _sp.run(["make", "-s", "-C", _HERE, "all"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not _os.path.exists(_LIB):
            build()
        L = _C.CDLL(_LIB)
        L.orc_negative_count.restype = _C.c_int
        L.orc_negative_count.argtypes = [_C.c_int, _C.c_void_p, _C.c_void_p, _C.c_double]
        L.orc_bisection.argtypes = [_C.c_int, _C.c_void_p, _C.c_void_p, _C.c_double, _C.c_double,
                                    _C.c_double, _C.c_int, _C.c_void_p, _C.c_void_p]
        L.orc_twisted_vectors.argtypes = [_C.c_int, _C.c_int, _C.c_void_p, _C.c_void_p, _C.c_void_p,
                                          _C.c_void_p, _C.c_void_p]
        L.orc_bidiagonal_svd.restype = _C.c_int
        L.orc_bidiagonal_svd.argtypes = [_C.c_int, _C.c_void_p, _C.c_void_p, _C.c_void_p,
                                         _C.c_void_p, _C.c_void_p, _C.c_int]
        L.orc_givens_tables.argtypes = [_C.c_size_t, _C.c_size_t, _C.c_int, _C.c_uint, _C.c_void_p,
                                        _C.c_void_p, _C.c_void_p]
        for f in (L.orc_givens_mask, L.orc_block_shift_mask):
            f.argtypes = [_C.c_size_t, _C.c_size_t, _C.c_size_t, _C.c_void_p, _C.c_int, _C.c_int,
                          _C.c_uint]
        L.orc_givens_variant.argtypes = [_C.c_size_t, _C.c_size_t, _C.c_size_t, _C.c_void_p, _C.c_int, _C.c_int,
                                         _C.c_uint, _C.c_int]
        for f in (L.orc_block_mask, L.orc_house_mask, L.orc_householder_reflector_mask):
            f.restype = _C.c_int
            f.argtypes = [_C.c_size_t, _C.c_size_t, _C.c_size_t, _C.c_void_p, _C.c_int, _C.c_int, _C.c_uint]
        L.orc_shuffle_block_mask.restype = _C.c_int
        L.orc_shuffle_block_mask.argtypes = [_C.c_size_t, _C.c_size_t, _C.c_size_t, _C.c_int, _C.c_void_p,
                                             _C.c_int, _C.c_int, _C.c_uint]
        L.orc_square_convert.argtypes = [_C.c_size_t, _C.c_void_p, _C.c_void_p, _C.c_void_p]
        L.orc_srand.argtypes = [_C.c_uint]
        L.orc_rand.restype = _C.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_C.c_void_p)


def _f64(a):
    return _np.ascontiguousarray(a, dtype=_np.float64)


def negative_count(alpha, beta, mu):
    a, b = _f64(alpha), _f64(beta if len(beta) else [0.0])
    return lib().orc_negative_count(len(a), _p(a), _p(b), float(mu))


def bisection(alpha, beta, lo, hi, tol=1e-20, top_k=None):
    a, b = _f64(alpha), _f64(beta if len(beta) else [0.0])
    n = len(a)
    top_k = n if top_k is None else top_k
    s = _np.zeros(max(n, 1))
    cnt = _C.c_int(0)
    lib().orc_bisection(n, _p(a), _p(b), lo, hi, tol, top_k, _p(s), _C.byref(cnt))
    return s[:cnt.value]


def twisted_vectors(alpha, beta, sigma):
    a, b, s = _f64(alpha), _f64(beta if len(beta) else [0.0]), _f64(sigma)
    n, c = len(a), len(s)
    U = _np.zeros((n, c))
    V = _np.zeros((c, n))
    lib().orc_twisted_vectors(n, c, _p(s), _p(a), _p(b), _p(U), _p(V))
    return U, V


def bidiagonal_svd(alpha, beta, top_k=None):
    """(sigma, U k x top_k, V top_k x k) as bbtsvd.cpp:932-968."""
    a, b = _f64(alpha), _f64(beta if len(beta) else [0.0])
    k = len(a)
    top_k = k if top_k is None else top_k
    U = _np.zeros((k, top_k))
    V = _np.zeros((top_k, k))
    s = _np.zeros(max(k, 1))
    rc = lib().orc_bidiagonal_svd(k, _p(a), _p(b), _p(U), _p(V), _p(s), top_k)
    if rc != 0:
        raise RuntimeError("bisection found fewer singular values than top_k")
    return s[:top_k], U, V


def givens_tables(k, passes, mask, seed):
    ops = (k + (k & 1)) // 2
    pr = _np.zeros((passes, ops, 2), dtype=_np.int32)
    c = _np.zeros((passes, ops))
    s = _np.zeros((passes, ops))
    lib().orc_givens_tables(k, passes, int(bool(mask)), seed, _p(pr), _p(c), _p(s))
    return pr, c, s


def givens_mask(x, passes, mask, is_left, seed):
    y = _f64(x).copy()
    m, n = y.shape
    lib().orc_givens_mask(m, n, passes, _p(y), int(bool(mask)), int(bool(is_left)), seed)
    return y


def givens_variant(x, passes, mask, is_left, seed, cached):
    """naive_givens_mask_parallel (cached=False) or
    givens_mask_cache_optimized_parallel (cached=True) on a copy of x."""
    y = _f64(x).copy()
    m, n = y.shape
    lib().orc_givens_variant(m, n, passes, _p(y), int(bool(mask)), int(bool(is_left)), seed, int(bool(cached)))
    return y


def dense_mask(kind, x, size, mask, is_left, seed, rounds=0):
    """block_mask / shuffle_block_mask / house_mask / householder_reflector_mask
    (kind "block", "shufblock", "house", "reflector") on a copy of x (m x n as
    the reference's buffer), over the LAPACK the process has loaded."""
    y = _f64(x).copy()
    m, n = y.shape
    L = lib()
    a = (m, n, size)
    t = (_p(y), int(bool(mask)), int(bool(is_left)), seed)
    if kind == "shufblock":
        rc = L.orc_shuffle_block_mask(*a, rounds, *t)
    else:
        rc = {"block": L.orc_block_mask, "house": L.orc_house_mask,
              "reflector": L.orc_householder_reflector_mask}[kind](*a, *t)
    if rc != 0:
        raise RuntimeError("no LAPACK loaded in this process")
    return y


def rand():
    """glibc's next rand() value (the state the restated masks leave behind)."""
    return lib().orc_rand()


def block_shift_mask(x, passes, mask, is_left, seed):
    y = _f64(x).copy()
    m, n = y.shape
    lib().orc_block_shift_mask(m, n, passes, _p(y), int(bool(mask)), int(bool(is_left)), seed)
    return y


def square_convert(k):
    r, c, rem = _C.c_size_t(), _C.c_size_t(), _C.c_size_t()
    lib().orc_square_convert(k, _C.byref(r), _C.byref(c), _C.byref(rem))
    return r.value, c.value, rem.value


def reference_seeds(seed, participants):
    """Mask seeds as the reference's participants derive them from the shared
    --seed: every process calls srand(seed) (client.cpp:196); participant 0
    draws the public seed (:498) and then its private seed (:531); every other
    participant's first draw is its private seed."""
    L = lib()
    L.orc_srand(seed)
    r1 = L.orc_rand() & 0xFFFFFFFF
    r2 = L.orc_rand() & 0xFFFFFFFF
    return r1, [r2] + [r1] * (participants - 1)
