"""The sign recovery of the split-precision local QRs (excalibur_b200/csrc/
chol.cu: householder_signs and its cooperative blocked form), restated in
numpy and checked against LAPACK on the CPU.

Householder QR of A = Q+ R+ (R+ with a positive diagonal) gives Q+ D, D =
diag(d), d_j = sign of dgeqrf's R_jj.  The compact-WY identity makes the
unpivoted LU of I - Q1 D (Q1 the top block of Q+) have pivots 1 + |c_j| >= 1,
where c_j is the j-th diagonal entry of Q1 once the earlier columns are
eliminated, so d_j = -sign(c_j).  The elimination runs on Q1 itself with the
multipliers l_ij = -d_j q_ij / (1 + |c_j|).

For a square A, LAPACK's last reflector is the identity (tau = 0, R_mm =
alpha): the last pivot is 0 and d_m = sign(c_m).  The pipeline's QRs are all
strictly tall (local_n > 5m, reduced global_n > m), so the library's kernels
implement the tall rule only; the square rule is checked here as a property
of dgeqrf."""
import numpy as np
import pytest
import scipy.linalg

LB = 16   # panel width of the blocked form


def sign_d(c, last_of_square):
    if last_of_square:
        return -1.0 if c < 0.0 else 1.0
    return 1.0 if c < 0.0 else -1.0


def signs_unblocked(Q1, square=False):
    A = Q1.copy()
    m = A.shape[1]
    d = np.empty(m)
    for j in range(m):
        c = A[j, j]
        d[j] = sign_d(c, square and j == m - 1)
        f = -d[j] / (1.0 + abs(c))
        l = f * A[j + 1:, j]
        A[j + 1:, j] = l
        A[j + 1:, j + 1:] -= np.outer(l, A[j, j + 1:])
    return d


def signs_blocked(Q1, square=False):
    """Right-looking with LB-column panels, as lu_sign_coop_kernel: factor a
    panel (the unblocked elimination on its rows), U12 = L11^-1 A12 (unit
    lower), A22 -= L21 U12."""
    A = Q1.copy()
    rows, m = A.shape
    d = np.empty(m)
    for p0 in range(0, m, LB):
        pb = min(LB, m - p0)
        P = A[p0:, p0:p0 + pb]   # a view: the panel, rows p0..
        for j in range(pb):
            c = P[j, j]
            d[p0 + j] = sign_d(c, square and p0 + j == m - 1)
            f = -d[p0 + j] / (1.0 + abs(c))
            l = f * P[j + 1:, j]
            P[j + 1:, j] = l
            P[j + 1:, j + 1:] -= np.outer(l, P[j, j + 1:])
        if p0 + pb < m:
            L11 = np.tril(A[p0:p0 + pb, p0:p0 + pb], -1) + np.eye(pb)
            A[p0:p0 + pb, p0 + pb:] = scipy.linalg.solve_triangular(L11, A[p0:p0 + pb, p0 + pb:], lower=True,
                                                                     unit_diagonal=True)
            A[p0 + pb:, p0 + pb:] -= A[p0 + pb:, p0:p0 + pb] @ A[p0:p0 + pb, p0 + pb:]
    return d


def block(n, m, cond, seed):
    rng = np.random.default_rng(seed)
    U, _ = np.linalg.qr(rng.standard_normal((n, m)))
    V, _ = np.linalg.qr(rng.standard_normal((m, m)))
    return (U * np.geomspace(1.0, 1.0 / cond, m)) @ V.T


@pytest.mark.parametrize("n,m,cond", [(200, 40, 1e2), (600, 100, 1e6), (300, 37, 1e3), (64, 64, 10.0)])
def test_signs_match_dgeqrf(n, m, cond):
    A = block(n, m, cond, n + m)
    R = scipy.linalg.qr(A, mode="r")[0][:m]           # dgeqrf
    d_ref = np.sign(np.diag(R))
    Q, Rq = np.linalg.qr(A)
    Qp = Q * np.sign(np.diag(Rq))                       # Q+ : R+ has a positive diagonal
    Q1 = Qp[:m]
    assert np.array_equal(signs_unblocked(Q1, n == m), d_ref)
    assert np.array_equal(signs_blocked(Q1, n == m), d_ref)


def test_pivots_are_at_least_one():
    A = block(400, 50, 1e4, 7)
    Q, Rq = np.linalg.qr(A)
    Q1 = (Q * np.sign(np.diag(Rq)))[:50].copy()
    d = signs_unblocked(Q1)
    # I - Q1 D = L U has U's diagonal 1 - d_j c_j = 1 + |c_j|: an unpivoted LU
    # of I - Q1 D succeeds with every pivot >= 1
    B = np.eye(50) - Q1 * d
    P, L, U = scipy.linalg.lu(B)
    LU = B.copy()
    for j in range(50):
        piv = LU[j, j]
        assert piv >= 1.0 - 1e-12
        LU[j + 1:, j] /= piv
        LU[j + 1:, j + 1:] -= np.outer(LU[j + 1:, j], LU[j, j + 1:])
