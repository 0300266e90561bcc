"""excalibur_b200 — Excalibur's matrix-factorisation hot path on B200 (sm_100a).

Python mirror of the reference's API (Excalibur include/bbtsvd.hpp and the
math inline in DecentralizedClient::run()), calling the CUDA kernels of
libexcalibur_b200.so through its C ABI (include/bbtsvd_b200.h).  Device
arrays are torch CUDA tensors (float64, contiguous); numpy arrays are copied
to the device and results copied back.  There is no CPU path: every method
raises if the library or a GPU is missing.

    ctx = Context(0)
    sigma, U, V = ctx.bidiagonal_bisection_twisted_svd(alpha, beta, top_k)
    ctx.block_shift_mask(x, 32, mask=True, is_left=True, seed=s)
    sigma, U, VT = ctx.fedsvd(blocks, public_seed, private_seeds)
"""
import ctypes as C
import os

import numpy as np

from ._lib import BBT_OK, STATUS, FedSVDConfig, load

__all__ = ["Context", "BBTError", "load", "reference_seeds"]


class BBTError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("excalibur_b200 needs a CUDA GPU (no CPU fallback)")
    return torch


def reference_seeds(seed, participants):
    """(public_seed, [private_seed]) as the reference's participants derive
    them from a shared --seed with glibc rand() (client.cpp:196, 498, 531):
    participant 0 draws the public seed then its private seed; every other
    participant's first draw is its private seed."""
    libc = C.CDLL("libc.so.6")
    libc.srand(C.c_uint(seed))
    r1 = libc.rand() & 0xFFFFFFFF
    r2 = libc.rand() & 0xFFFFFFFF
    return r1, [r2] + [r1] * (participants - 1)


class Context:
    """A bbt_ctx: one CUDA stream, a device workspace, error text."""

    def __init__(self, device=0):
        self.torch = _torch()
        self.L = load()
        self.device = device
        self.torch.cuda.set_device(device)
        h = C.c_void_p()
        self._check(self.L.bbt_create(C.byref(h), device), "bbt_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.bbt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- helpers -----------------------------------------------------------
    def _check(self, st, what):
        if st != BBT_OK:
            msg = self.L.bbt_last_error(self.h).decode() if getattr(self, "h", None) else what
            raise BBTError(st, f"{what}: {msg}")

    def _dev(self, x, dtype=None):
        """torch CUDA float64 contiguous tensor (copy of numpy input)."""
        t = self.torch
        dtype = dtype or t.float64
        if isinstance(x, t.Tensor):
            assert x.is_cuda and x.dtype == dtype and x.is_contiguous(), "need a contiguous CUDA tensor"
            return x
        return t.as_tensor(np.ascontiguousarray(x), dtype=dtype, device=f"cuda:{self.device}")

    def _empty(self, *shape, dtype=None):
        t = self.torch
        return t.empty(*shape, dtype=dtype or t.float64, device=f"cuda:{self.device}")

    def sync(self):
        self._check(self.L.bbt_synchronize(self.h), "synchronize")

    def launches(self):
        return int(self.L.bbt_kernel_launches(self.h))

    @staticmethod
    def _p(t):
        return C.c_void_p(t.data_ptr())

    def _pre(self):
        self.torch.cuda.synchronize(self.device)   # inputs written by torch are complete

    def set_stream(self, stream=None):
        """Launch on a borrowed CUDA stream (a torch.cuda.Stream or a raw
        cudaStream_t handle); None returns to the context's own stream."""
        h = None if stream is None else getattr(stream, "cuda_stream", stream)
        self._check(self.L.bbt_set_stream(self.h, C.c_void_p(h) if h else None), "set_stream")

    # -- bbtsvd.hpp ---------------------------------------------------------
    def negative_count(self, alpha, beta, mu):
        """Sturm counts at every shift in mu (bbtsvd.cpp:7-17)."""
        a, b = self._dev(alpha), self._dev(beta if len(beta) else np.zeros(1))
        mus = self._dev(np.atleast_1d(np.asarray(mu, dtype=np.float64)))
        out = self._empty(mus.numel(), dtype=self.torch.int32)
        self._pre()
        self._check(self.L.bbt_negative_count(self.h, a.numel(), self._p(a), self._p(b), self._p(mus),
                                              mus.numel(), self._p(out)), "negative_count")
        self.sync()
        return out.cpu().numpy()

    def bisection_singular_values(self, alpha, beta, lo, hi, tol=1e-20, top_k=None):
        """Singular values by the reference's bisection tree (bbtsvd.cpp:19-52)."""
        a, b = self._dev(alpha), self._dev(beta if len(beta) else np.zeros(1))
        n = a.numel()
        top_k = n if top_k is None else top_k
        s = self._empty(max(n, 1))
        cnt = C.c_int(0)
        self._pre()
        self._check(self.L.bbt_bisection(self.h, n, self._p(a), self._p(b), lo, hi, tol, top_k, self._p(s),
                                         C.byref(cnt)), "bisection")
        self.sync()
        return s[: cnt.value]

    def two_side_singular_vectors_twisted_factorization(self, alpha, beta, sigma):
        """(U n x cnt, V cnt x n) for given singular values (bbtsvd.cpp:138-147)."""
        a, b = self._dev(alpha), self._dev(beta if len(beta) else np.zeros(1))
        s = self._dev(sigma)
        n, c = a.numel(), s.numel()
        U = self._empty(n, c)
        V = self._empty(c, n)
        self._pre()
        self._check(self.L.bbt_twisted_vectors(self.h, n, c, self._p(s), self._p(a), self._p(b), self._p(U),
                                               self._p(V)), "twisted_vectors")
        self.sync()
        return U, V

    def bidiagonal_bisection_twisted_svd(self, alpha, beta, top_k=None):
        """(sigma, U k x top_k, V top_k x k) (bbtsvd.cpp:932-968)."""
        a, b = self._dev(alpha), self._dev(beta if len(beta) else np.zeros(1))
        k = a.numel()
        top_k = k if top_k is None else top_k
        U = self._empty(k, top_k)
        V = self._empty(top_k, k)
        s = self._empty(top_k)
        self._pre()
        self._check(self.L.bbt_bidiagonal_svd(self.h, k, self._p(a), self._p(b), self._p(U), self._p(V),
                                              self._p(s), top_k), "bidiagonal_svd")
        self.sync()
        return s, U, V

    def givens_mask_cache_optimized_parallel_with_simd(self, x, mask_times, mask, is_left, seed):
        """In place on x (m x n row-major CUDA tensor) (bbtsvd.cpp:727-876)."""
        x = self._dev(x) if not isinstance(x, self.torch.Tensor) else x
        m, n = x.shape
        self._pre()
        self._check(self.L.bbt_givens_mask(self.h, m, n, mask_times, self._p(x), int(bool(mask)),
                                           int(bool(is_left)), seed), "givens_mask")
        self.sync()
        return x

    def block_shift_mask(self, x, mask_times, mask, is_left, seed):
        """In place on x (m x n row-major CUDA tensor) (bbtsvd.cpp:533-669)."""
        x = self._dev(x) if not isinstance(x, self.torch.Tensor) else x
        m, n = x.shape
        self._pre()
        self._check(self.L.bbt_block_shift_mask(self.h, m, n, mask_times, self._p(x), int(bool(mask)),
                                                int(bool(is_left)), seed), "block_shift_mask")
        self.sync()
        return x

    # -- client.cpp -----------------------------------------------------------
    def local_qr_reduction(self, x, compute_q=True):
        """Householder QR of X^T for X (m x local_n row-major, CUDA tensor,
        overwritten by Q^T when compute_q).  Returns R^T (m x m)
        (client.cpp:417-445)."""
        m, n = x.shape
        rt = self._empty(m, m)
        self._pre()
        self._check(self.L.bbt_local_qr(self.h, m, n, self._p(x), self._p(rt), int(bool(compute_q))), "local_qr")
        self.sync()
        return rt

    # -- learned bisection brackets (mlp.cu) ------------------------------------
    def gebrd(self, A):
        """Householder bidiagonalisation of a dense n x n matrix held
        column-major (a CUDA tensor holding X^T; overwritten).  Returns (d, e)."""
        n = A.shape[0]
        d, e = self._empty(n), self._empty(n)
        self._pre()
        self._check(self.L.bbt_gebrd(self.h, n, self._p(A), self._p(d), self._p(e)), "gebrd")
        self.sync()
        return d, e[: n - 1]

    def bidiagonal_singular_values(self, alpha, beta, brackets=None, top_k=None):
        """The reference's bisection on [0, ||a||^2 + ||b||^2] with tol 1e-20
        (bbtsvd.cpp:936-940); with brackets (count x 2, descending), the
        learned-bracket variant.  Returns sigma (or (sigma, stats))."""
        a, b = self._dev(alpha), self._dev(beta if len(beta) else np.zeros(1))
        n = a.numel()
        bound = float((a * a).sum() + ((b[: n - 1] * b[: n - 1]).sum() if n > 1 else 0.0))
        top_k = n if top_k is None else top_k
        if brackets is None:
            return self.bisection_singular_values(a, b, 0.0, bound, 1e-20, top_k)
        s = self._empty(max(n, 1))
        cnt = C.c_int(0)
        st = (C.c_longlong * 4)()
        br = self._dev(brackets)
        self._pre()
        self._check(self.L.bbt_bisection_bracketed(self.h, n, self._p(a), self._p(b), 0.0, bound, 1e-20, top_k,
                                                   self._p(br), self._p(s), C.byref(cnt), st), "bisection_bracketed")
        self.sync()
        return s[: cnt.value], {"sturm_evals": st[0], "rounds": st[1], "jumps": st[2], "verify_evals": st[3]}

    def bisection_stats(self):
        st = (C.c_longlong * 4)()
        self._check(self.L.bbt_bisection_stats(self.h, st), "bisection_stats")
        return {"sturm_evals": st[0], "rounds": st[1], "jumps": st[2], "verify_evals": st[3]}

    def mlp_param_count(self):
        return int(self.L.bbt_mlp_param_count())

    def mlp_features(self, alpha, beta, count=None):
        a, b = self._dev(alpha), self._dev(beta if len(beta) else np.zeros(1))
        k = a.numel()
        count = k if count is None else count
        X = self._empty(count, 10)
        self._pre()
        self._check(self.L.bbt_mlp_features(self.h, k, self._p(a), self._p(b), count, self._p(X)), "mlp_features")
        self.sync()
        return X

    def mlp_forward(self, X, theta):
        X, theta = self._dev(X), self._dev(theta)
        out = self._empty(X.shape[0], 2)
        self._pre()
        self._check(self.L.bbt_mlp_forward(self.h, X.shape[0], self._p(X), self._p(theta), self._p(out)),
                    "mlp_forward")
        self.sync()
        return out

    def mlp_grad(self, X, y, theta, grad=None, loss=None):
        """Mean Gaussian-NLL loss and its gradient over the batch (device)."""
        X, y, theta = self._dev(X), self._dev(y), self._dev(theta)
        grad = self._empty(theta.numel()) if grad is None else grad
        loss = self._empty(1) if loss is None else loss
        self._pre()
        self._check(self.L.bbt_mlp_grad(self.h, X.shape[0], self._p(X), self._p(y), self._p(theta), self._p(grad),
                                        self._p(loss)), "mlp_grad")
        self.sync()
        return grad, loss

    def mlp_adam(self, theta, grad, m, v, lr, step):
        self._pre()
        self._check(self.L.bbt_mlp_adam(self.h, self._p(theta), self._p(grad), self._p(m), self._p(v), lr, step),
                    "mlp_adam")
        self.sync()

    def mlp_brackets(self, alpha, beta, theta, count=None, z=3.0):
        a, b = self._dev(alpha), self._dev(beta if len(beta) else np.zeros(1))
        k = a.numel()
        count = k if count is None else count
        theta = self._dev(theta)
        br = self._empty(count, 2)
        self._pre()
        self._check(self.L.bbt_mlp_brackets(self.h, k, self._p(a), self._p(b), count, self._p(theta), z,
                                            self._p(br)), "mlp_brackets")
        self.sync()
        return br

    def set_bracket_model(self, theta=None, z=3.0):
        """Use the learned brackets inside every bisection of this context
        (theta: numpy parameters; None switches them off)."""
        if theta is None:
            self._check(self.L.bbt_set_bracket_model(self.h, None, z), "set_bracket_model")
            return
        th = np.ascontiguousarray(theta, dtype=np.float64)
        assert th.size == self.mlp_param_count()
        self._check(self.L.bbt_set_bracket_model(self.h, th.ctypes.data_as(C.c_void_p), z), "set_bracket_model")

    def rademacher(self, N, n, seed):
        """S (N x n, +-1 in bf16; returned as an int16 tensor of bf16 bit
        patterns, row pitch n rounded up to 8)."""
        pitch = (n + 7) // 8 * 8
        S = self._empty(N, pitch, dtype=self.torch.int16)
        self._pre()
        self._check(self.L.bbt_rademacher(self.h, N, n, seed, self._p(S)), "rademacher")
        self.sync()
        return S

    def sketch_bf16x3(self, x, S, N):
        """Y (m x N) = X S^T for X (m x n, CUDA float64) on the tensor cores
        (BF16x3 pieces of X, FP32 accumulation per K-chunk)."""
        m, n = x.shape
        Y = self._empty(m, N)
        self._pre()
        self._check(self.L.bbt_sketch_bf16x3(self.h, m, n, self._p(x), N, self._p(S), self._p(Y)), "sketch_bf16x3")
        self.sync()
        return Y

    def mixed_local_qr(self, x, want_w=True):
        """Precision-1 local QR of X (m x local_n, CUDA float64, overwritten
        by Q_p^T).  Returns (R as an m x m tensor holding the column-major
        upper-triangular R, i.e. R^T row-major; W likewise, or None) with
        X^T = Q_p W R and Q_p W orthonormal."""
        m, n = x.shape
        R = self._empty(m, m)
        W = self._empty(m, m) if want_w else None
        self._pre()
        self._check(self.L.bbt_mixed_local_qr(self.h, m, n, self._p(x), self._p(R),
                                              self._p(W) if W is not None else None), "mixed_local_qr")
        self.sync()
        return R, W

    def _config(self, m, local_n, public_seed, private_seeds, top_k, svd_mode, precision, labels=None):
        P = len(local_n)
        self._ln = (C.c_size_t * P)(*local_n)
        self._ps = (C.c_uint * P)(*[s & 0xFFFFFFFF for s in private_seeds])
        return FedSVDConfig(P, m, self._ln, public_seed & 0xFFFFFFFF, self._ps, top_k, svd_mode, precision,
                            labels)

    @staticmethod
    def _shapes(blocks, tall):
        """(m, [local_n]) of the blocks in the branch's layout: X_c (m x
        local_n) short-and-wide, X_c^T (local_n x m) tall-and-skinny."""
        if tall:
            m, ln = blocks[0].shape[1], [b.shape[0] for b in blocks]
            if m <= sum(ln):
                raise ValueError(f"tall layout needs m={m} > global_n={sum(ln)}")
        else:
            m, ln = blocks[0].shape[0], [b.shape[1] for b in blocks]
            if m > sum(ln):
                raise ValueError(f"m={m} > global_n={sum(ln)}: pass the blocks transposed with tall=True")
        return m, ln

    @staticmethod
    def _outputs(U, VT, m, ln, k, svd_mode, tall):
        if svd_mode in (3, 4):
            Uo = None
        else:
            Uo = U[: m * k].reshape(k, m) if tall else U[: m * k].reshape(m, k)
        if svd_mode == 2:
            VTo = None
        elif svd_mode == 4:
            VTo = [v[:n] for v, n in zip(VT, ln)]
        else:
            VTo = [v[: k * n].reshape(k, n) for v, n in zip(VT, ln)]
        return Uo, VTo

    def fedsvd(self, blocks, public_seed, private_seeds, top_k=-1, svd_mode=1, precision=0, tall=False,
               labels=None):
        """DecentralizedClient::run() for P participants on this GPU
        (client.cpp:447-1200).  blocks (CUDA tensors, overwritten): m x
        local_n each, or with tall=True (m > global_n) local_n x m each, the
        reference's layout in its tall-and-skinny branch.  Returns (sigma k,
        FinalU, [FinalVT_c k x local_n]); FinalU is m x k (k x m with tall),
        None in svd_modes 3 and 4; the FinalVT list is None in svd_mode 2.
        svd_mode 4 (linear regression, tall only) takes labels (CUDA tensor,
        m) and returns [w_c (local_n)] in place of FinalVT."""
        P = len(blocks)
        m, ln = self._shapes(blocks, tall)
        kmax = min(m, sum(ln))
        y = labels.contiguous() if labels is not None else None
        cfg = self._config(m, ln, public_seed, private_seeds, top_k, svd_mode, precision,
                           C.c_void_p(y.data_ptr()) if y is not None else None)
        sig = self._empty(kmax)
        U = self._empty(m * kmax)
        VT = [self._empty(m * n) for n in ln]
        bp = (C.c_void_p * P)(*[b.data_ptr() for b in blocks])
        vp = (C.c_void_p * P)(*[v.data_ptr() for v in VT])
        k = C.c_int(0)
        self._pre()
        self._check(self.L.bbt_fedsvd_run(self.h, C.byref(cfg), bp, self._p(sig), self._p(U), vp, C.byref(k)),
                    "fedsvd")
        self.sync()
        k = k.value
        Uo, VTo = self._outputs(U, VT, m, ln, k, svd_mode, tall)
        return sig[:k], Uo, VTo

    def fedsvd_tune(self, m, local_n, top_k=-1, svd_mode=1, precision=0):
        """Autotune the batched local QR for these shapes and precision mode
        (kept in the context).  Returns (streams, panel width, ms)."""
        cfg = self._config(m, list(local_n), 0, [0] * len(local_n), top_k, svd_mode, precision)
        st, nb, ms = C.c_int(), C.c_int(), C.c_double()
        self._pre()
        self._check(self.L.bbt_fedsvd_tune(self.h, C.byref(cfg), C.byref(st), C.byref(nb), C.byref(ms)),
                    "fedsvd_tune")
        return st.value, nb.value, ms.value

    def fedsvd_host(self, blocks, public_seed, private_seeds, top_k=-1, svd_mode=1, precision=0, out=None,
                    tall=False, labels=None):
        """Same through the host-pointer entry (bbt_fedsvd_run_host): numpy
        blocks (and labels) in, numpy results out (copies timed inside the
        call)."""
        P = len(blocks)
        m, ln = self._shapes(blocks, tall)
        kmax = min(m, sum(ln))
        y = np.ascontiguousarray(labels, dtype=np.float64) if labels is not None else None
        cfg = self._config(m, ln, public_seed, private_seeds, top_k, svd_mode, precision,
                           C.c_void_p(y.ctypes.data) if y is not None else None)
        blocks = [np.ascontiguousarray(b, dtype=np.float64) for b in blocks]
        if out is None:
            out = (np.empty(kmax), np.empty(m * kmax), [np.empty(m * n) for n in ln])
        sig, U, VT = out
        bp = (C.c_void_p * P)(*[b.ctypes.data for b in blocks])
        vp = (C.c_void_p * P)(*[v.ctypes.data for v in VT])
        k = C.c_int(0)
        self._check(self.L.bbt_fedsvd_run_host(self.h, C.byref(cfg), bp, C.c_void_p(sig.ctypes.data),
                                               C.c_void_p(U.ctypes.data), vp, C.byref(k)), "fedsvd_host")
        k = k.value
        Uo, VTo = self._outputs(U, VT, m, ln, k, svd_mode, tall)
        return sig[:k], Uo, VTo

    def fedsvd_files(self, dpath, m, local_n, public_seed, private_seeds, top_k=-1, svd_mode=1, precision=0,
                     out=None):
        """The pipeline on the reference's on-disk input (bbt_fedsvd_run_files):
        dpath/Client<c>.mat (m * local_n[c] float64 in the branch's layout,
        see excalibur_b200.datafiles) and, in svd_mode 4, dpath/y.mat.
        Returns numpy results as fedsvd_host."""
        P = len(local_n)
        ln = [int(n) for n in local_n]
        tall = m > sum(ln)
        kmax = min(m, sum(ln))
        cfg = self._config(m, ln, public_seed, private_seeds, top_k, svd_mode, precision)
        if out is None:
            out = (np.empty(kmax), np.empty(m * kmax), [np.empty(m * n) for n in ln])
        sig, U, VT = out
        vp = (C.c_void_p * P)(*[v.ctypes.data for v in VT])
        k = C.c_int(0)
        self._check(self.L.bbt_fedsvd_run_files(self.h, C.byref(cfg), os.fsencode(dpath), C.c_void_p(sig.ctypes.data),
                                                C.c_void_p(U.ctypes.data), vp, C.byref(k)), "fedsvd_files")
        k = k.value
        Uo, VTo = self._outputs(U, VT, m, ln, k, svd_mode, tall)
        return sig[:k], Uo, VTo

    def dgemm(self, transa, transb, A, B, alpha=1.0, beta=0.0, C=None):
        """C = alpha op(A) op(B) + beta C on column-major data.  A, B, C are
        CUDA tensors holding column-major matrices as their transposes
        (a column-major M x K matrix is a row-major K x M tensor)."""
        M = A.shape[0] if transa else A.shape[1]
        K = A.shape[1] if transa else A.shape[0]
        N = B.shape[0] if not transb else B.shape[1]
        K2 = B.shape[1] if not transb else B.shape[0]
        assert K == K2, (K, K2)
        if C is None:
            C = self._empty(N, M)
        self._pre()
        self._check(self.L.bbt_dgemm(self.h, int(transa), int(transb), M, N, K, alpha, self._p(A), A.shape[1],
                                     self._p(B), B.shape[1], beta, self._p(C), C.shape[1]), "dgemm")
        self.sync()
        return C

    def dgemm_crt(self, A, B, alpha=1.0, beta=0.0, C=None, bits=53):
        """C (M x N) = alpha A^T B + beta C for column-major A (K x M) and B
        (K x N) -- row-major tensors of M x K and N x K -- from exact integer
        products on the int8 tensor cores (operand rows rounded to `bits`
        bits).  C is returned as a row-major N x M tensor (its column-major
        transpose), as dgemm does."""
        M, K = A.shape
        N, K2 = B.shape
        assert K == K2, (K, K2)
        if C is None:
            C = self._empty(N, M)
        self._pre()
        self._check(self.L.bbt_dgemm_crt(self.h, M, N, K, alpha, self._p(A), A.shape[1], self._p(B), B.shape[1], beta,
                                         self._p(C), C.shape[1], bits), "dgemm_crt")
        self.sync()
        return C

    def gram_dd(self, X):
        """Upper triangle of G = X X^T (X row-major m x n, CUDA float64) as a
        double-double (Gh, Gl), each a row-major m x m tensor holding the
        column-major matrix (entries strictly below the diagonal undefined)."""
        m, n = X.shape
        Gh, Gl = self._empty(m, m), self._empty(m, m)
        self._pre()
        self._check(self.L.bbt_gram_dd(self.h, m, n, self._p(X), X.shape[1], self._p(Gh), self._p(Gl)), "gram_dd")
        self.sync()
        return Gh, Gl

    def exact_local_qr(self, X):
        """Exact-Gram QR of A = X^T (X row-major m x local_n CUDA float64,
        kept): returns (R, W, Rp, scale), R m x m with dgeqrf's row signs, all
        as row-major tensors holding the column-major matrices (R.T is R)."""
        m, n = X.shape
        R, W, Rp = self._empty(m, m), self._empty(m, m), self._empty(m, m)
        sc = self._empty(m)
        self._pre()
        self._check(self.L.bbt_exact_local_qr(self.h, m, n, self._p(X), self._p(R), self._p(W), self._p(Rp),
                                              self._p(sc)), "exact_local_qr")
        self.sync()
        return R, W, Rp, sc

    def exact_apply_q(self, X, scale, Rp, Z):
        """C = A_int Rp^-1 Z (rows x k) for the integers of A = X^T; Z is a
        row-major k x m tensor holding the column-major m x k matrix.
        Returns C as a row-major k x rows tensor (column-major rows x k)."""
        m, n = X.shape
        k = Z.shape[0]
        Cout = self._empty(k, n)
        self._pre()
        self._check(self.L.bbt_exact_apply_q(self.h, m, n, self._p(X), X.shape[1], self._p(scale), self._p(Rp),
                                             self._p(Z), k, self._p(Cout), n), "exact_apply_q")
        self.sync()
        return Cout

    def dgemm_ozaki(self, transa, transb, A, B, alpha=1.0, beta=0.0, C=None, upper=False):
        """dgemm's contract (same tensor conventions) computed from exact int8
        slices on the tensor cores (FP64-accurate)."""
        M = A.shape[0] if transa else A.shape[1]
        K = A.shape[1] if transa else A.shape[0]
        N = B.shape[0] if not transb else B.shape[1]
        K2 = B.shape[1] if not transb else B.shape[0]
        assert K == K2, (K, K2)
        if C is None:
            C = self.torch.zeros(N, M, dtype=self.torch.float64, device=f"cuda:{self.device}")
        self._pre()
        self._check(self.L.bbt_dgemm_ozaki(self.h, int(transa), int(transb), M, N, K, alpha, self._p(A), A.shape[1],
                                           self._p(B), B.shape[1], beta, self._p(C), C.shape[1], int(upper)),
                    "dgemm_ozaki")
        self.sync()
        return C

    def profile(self, enable=True):
        self._check(self.L.bbt_profile(self.h, int(bool(enable))), "profile")

    def profile_get(self):
        """{class: (ms, launches, work)} since profiling was switched on."""
        from ._lib import PROF_CLASSES
        out = {}
        for i, name in enumerate(PROF_CLASSES):
            ms, n, w = C.c_double(), C.c_uint64(), C.c_double()
            self._check(self.L.bbt_profile_get(self.h, i, C.byref(ms), C.byref(n), C.byref(w)), "profile_get")
            out[name] = (ms.value, n.value, w.value)
        return out

    def svd_dense(self, X, top_k=-1):
        """SVD of a dense m x m matrix (CUDA tensor, overwritten) by Ralha
        bidiagonalisation + bisection + twisted vectors + back-transforms.
        Returns (sigma k, U m x k, VT k x m)."""
        m = X.shape[0]
        assert X.shape == (m, m)
        sig = self._empty(m)
        U = self._empty(m * m)
        VT = self._empty(m * m)
        k = C.c_int(0)
        self._pre()
        self._check(self.L.bbt_svd_dense(self.h, m, self._p(X), top_k, self._p(sig), self._p(U), self._p(VT),
                                         C.byref(k)), "svd_dense")
        self.sync()
        k = k.value
        return sig[:k], U[: m * k].view(m, k), VT[: k * m].view(k, m)

    def stage_ms(self):
        """Per-phase ms of the last fedsvd: local_qr, apply_mask, global_qr,
        bi_diag, bsvd, combine_svd_remove_mask (the reference's timers)."""
        buf = (C.c_double * 6)()
        self._check(self.L.bbt_fedsvd_stage_ms(self.h, buf, 6), "stage_ms")
        return dict(zip(("local_qr", "apply_mask", "global_qr", "bi_diag", "bsvd", "combine_svd_remove_mask"),
                        list(buf)))
