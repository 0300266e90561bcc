"""bbt_twisted_vectors_noalloc: the twisted-vector entry point for callers
that must not allocate device memory (for example an allocation-free hot
loop, or a process whose device memory belongs to another allocator).  It
keeps its work arrays in a static device array instead of calling
cudaMalloc.  Checked here through the C ABI against bbt_twisted_vectors, the
allocating entry point, on two calls in a row with different shapes (the
shared array keeps the first call's contents).  This file is collected last
so a failure here leaves every other test already run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


SCRATCH_DOUBLES = (64 << 20) // 8   # the static array: 64 MiB


def _need(n, cnt):
    """Doubles of the static array a call of shape (n, cnt) uses: 2n + 6(n+1)cnt + n cnt
    plus one byte per vector, each array rounded up to 256 bytes."""
    up = lambda d: (d + 31) & ~31
    return 2 * up(n) + 6 * up((n + 1) * cnt) + up(n * cnt) + up((cnt + 7) // 8)


def _largest_square():
    n = 1
    while _need(n + 1, n + 1) <= SCRATCH_DOUBLES:
        n += 1
    return n


def _case(seed, n, cnt):
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.5, 2.0, n)
    b = rng.uniform(-1.0, 1.0, n - 1)
    B = np.diag(a) + np.diag(b, 1)
    s = np.linalg.svd(B, compute_uv=False)[:cnt].copy()
    return a, b, s


def test_noalloc_twisted_matches_allocating_entry():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from excalibur_b200 import _lib
    L = _lib.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    h = C.c_void_p()
    assert L.bbt_create(C.byref(h), 0) == 0
    try:
        for seed, n, cnt in ((1, 300, 300), (2, 257, 100)):
            a, b, s = _case(seed, n, cnt)
            da = torch.as_tensor(a, device=dev)
            db = torch.as_tensor(b, device=dev)
            ds = torch.as_tensor(s, device=dev)
            U0 = torch.empty(n, cnt, dtype=torch.float64, device=dev)
            V0 = torch.empty(cnt, n, dtype=torch.float64, device=dev)
            U1 = torch.full((n, cnt), np.nan, dtype=torch.float64, device=dev)
            V1 = torch.full((cnt, n), np.nan, dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            p = lambda t: C.c_void_p(t.data_ptr())
            assert L.bbt_twisted_vectors(h, n, cnt, p(ds), p(da), p(db), p(U0), p(V0)) == 0
            assert L.bbt_synchronize(h) == 0
            st = L.bbt_twisted_vectors_noalloc(None, n, cnt, p(ds), p(da), p(db), p(U1), p(V1))
            assert st == 0
            torch.cuda.synchronize()
            # same kernels, same arithmetic: the tolerance of the other twisted-vector tests
            assert torch.max(torch.abs(U1 - U0)).item() <= 1e-15
            assert torch.max(torch.abs(V1 - V0)).item() <= 1e-15
        # the largest square shape the static array holds runs and matches; one more is rejected
        # before any GPU work
        n_fit = _largest_square()
        assert _need(n_fit, n_fit) <= SCRATCH_DOUBLES < _need(n_fit + 1, n_fit + 1)
        a, b, s = _case(3, n_fit, n_fit)
        da, db, ds = (torch.as_tensor(v, device=dev) for v in (a, b, s))
        U0 = torch.empty(n_fit, n_fit, dtype=torch.float64, device=dev)
        V0 = torch.empty(n_fit, n_fit, dtype=torch.float64, device=dev)
        U1 = torch.empty_like(U0)
        V1 = torch.empty_like(V0)
        torch.cuda.synchronize()
        assert L.bbt_twisted_vectors(h, n_fit, n_fit, p(ds), p(da), p(db), p(U0), p(V0)) == 0
        assert L.bbt_synchronize(h) == 0
        # the property the entry exists for: a warmed-up call leaves the device's free memory unchanged
        free0 = torch.cuda.mem_get_info(dev)[0]
        assert L.bbt_twisted_vectors_noalloc(None, n_fit, n_fit, p(ds), p(da), p(db), p(U1), p(V1)) == 0
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info(dev)[0] == free0
        assert torch.max(torch.abs(U1 - U0)).item() <= 1e-15
        assert torch.max(torch.abs(V1 - V0)).item() <= 1e-15
        big = n_fit + 1
        da = torch.as_tensor(np.ones(big), device=dev)
        db = torch.as_tensor(np.ones(big - 1), device=dev)
        ds = torch.as_tensor(np.ones(big), device=dev)
        U = torch.empty(big * big, dtype=torch.float64, device=dev)
        assert L.bbt_twisted_vectors_noalloc(None, big, big, p(ds), p(da), p(db), p(U), p(U)) == 1
    finally:
        L.bbt_destroy(h)
