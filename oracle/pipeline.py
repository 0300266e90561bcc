"""ORACLE — test infrastructure, not product code.

numpy restatement of Excalibur's ``DecentralizedClient::run()``: the
short-and-wide branch (m <= global_n, ``src/client.cpp:570-606, 680-1199``,
``run``) and the tall-and-skinny branch with its linear-regression mode
(m > global_n, ``src/client.cpp:543-568, 627-679, 1002-1169``, ``run_tall``),
with all P participants held in one process.  The reference's socket
collectives become plain array operations; its ``ring_all_reduce_sum``
becomes a sum over participants in index order.

Conventions (as in the reference): participant c holds X_c, a row-major
m x local_n[c] float64 block; the global matrix is X = [X_0 | X_1 | ...].
Outputs: sigma (descending), FinalU (m x k, row-major, every participant
holds the same), FinalVT_c (k x local_n[c]) per participant, with
X ~= FinalU diag(sigma) [FinalVT_0 | FinalVT_1 | ...].
"""
import numpy as np
import scipy.linalg.lapack as lapack

from . import bidiagonal_svd, block_shift_mask, negative_count

LOCAL_QR_THRESHOLD = 5.0   # client.cpp:482
MASK_PASSES = 32           # client.cpp:536


def row_split(m, P):
    """m_part / m_part_pos (client.cpp:613-624)."""
    part = [m // P + (1 if i < m % P else 0) for i in range(P)]
    pos = [0]
    for p in part:
        pos.append(pos[-1] + p)
    return part, pos


def reduced_width(m, local_n):
    """Columns kept after the local QR: min(m, local_n) when the integer
    ratio local_n/m exceeds 5 (client.cpp:505,510,517)."""
    return min(m, local_n) if (local_n // m) > LOCAL_QR_THRESHOLD else local_n


def local_qr(x):
    """local_qr_reduction(local_n, m, ...) with compute_q (client.cpp:417-445):
    dgeqrf of A = X_c^T (local_n x m, column-major = X_c row-major), Q by
    dorgqr.  Returns (R^T as the new m x m block, Q^T as m x local_n)."""
    A = np.asfortranarray(x.T)
    qr, tau, _, info = lapack.dgeqrf(A)
    assert info == 0
    R = np.triu(qr[: x.shape[0], :])
    Q, _, info = lapack.dorgqr(qr, tau)
    assert info == 0
    return R.T.copy(), np.ascontiguousarray(Q.T)


def householder(alpha, x):
    """dlarfg: H (alpha; x) = (beta; 0), H = I - tau (1; v)(1; v)^T."""
    xn = np.linalg.norm(x)
    if xn == 0.0:
        return alpha, np.zeros_like(x), 0.0
    beta = -np.copysign(np.hypot(alpha, xn), alpha)
    tau = (beta - alpha) / beta
    return beta, x / (alpha - beta), tau


def drotg(a, b):
    """Reference-BLAS drotg: returns (r, c, s) with r carrying the sign of
    the larger-magnitude input."""
    roe = b if abs(b) > abs(a) else a
    scale = abs(a) + abs(b)
    if scale == 0.0:
        return 0.0, 1.0, 0.0
    r = scale * np.sqrt((a / scale) ** 2 + (b / scale) ** 2)
    r = np.copysign(1.0, roe) * r
    return r, a / r, b / r


def ralha(slabs):
    """One-sided (Ralha) bidiagonalisation, overlapped variant
    (client.cpp:829-910), of the m x m matrix whose column slabs are
    ``slabs`` (participant c holds m x m_part[c]).  Returns lower-bidiagonal
    alpha, beta, the Householder store (m x m, reflector j in column j from
    row j, unit diagonal), tau (m), and the left vectors as per-participant
    slabs (m x m_part[c])."""
    W = [s.copy() for s in slabs]
    m = W[0].shape[0]
    house = np.zeros((m, m))
    house[0, 0] = 1.0
    tau = np.zeros(m)
    alpha = np.zeros(m)
    beta = np.zeros(max(m - 1, 1))
    V = [np.zeros_like(w) for w in W]
    alpha[0] = np.sqrt(sum(float(w[0] @ w[0]) for w in W))
    for c in range(len(W)):
        V[c][0] = W[c][0] / alpha[0]
    for i in range(m - 2):
        msg = np.zeros(m + 3 - i)
        for w, v in zip(W, V):               # fixed-order in-process all-reduce
            part = np.zeros(m + 3 - i)
            part[: m - 1 - i] = w[i + 1:] @ w[i]
            if i > 0:
                part[m - i - 1] = w[i] @ v[i - 1]
                part[m - i] = v[i - 1] @ v[i - 1]
                part[m - i + 1] = w[i] @ w[i]
                part[m - i + 2] = v[i - 1] @ w[i]
            msg += part
        g = msg[: m - 1 - i]
        if i > 0:
            beta[i - 1] = msg[m - i - 1]
        _, vec, t = householder(g[0], g[1:])
        house[i + 1, i + 1] = 1.0
        house[i + 2:, i + 1] = vec
        tau[i + 1] = t
        h = house[i + 1:, i + 1]
        for c in range(len(W)):
            blk = W[c][i + 1:]
            W[c][i + 1:] = blk - t * np.outer(h, h @ blk)
        if i > 0:
            b = beta[i - 1]
            for c in range(len(W)):
                W[c][i] = W[c][i] - b * V[c][i - 1]
            alpha[i] = np.sqrt(msg[m - i] * b * b + msg[m - i + 1] - 2 * b * msg[m - i + 2])
            for c in range(len(W)):
                V[c][i] = W[c][i] / alpha[i]
    for i in range(max(m - 2, 1), m):        # tail steps (client.cpp:897-905)
        if i < 1:
            continue
        b = sum(float(w[i] @ v[i - 1]) for w, v in zip(W, V))
        beta[i - 1] = b
        for c in range(len(W)):
            W[c][i] = W[c][i] - b * V[c][i - 1]
        alpha[i] = np.sqrt(sum(float(w[i] @ w[i]) for w in W))
        for c in range(len(W)):
            V[c][i] = W[c][i] / alpha[i]
    return alpha, beta[: m - 1], house, tau, V


def lower_to_upper(alpha, beta):
    """drotg sweep turning the lower bidiagonal upper (client.cpp:947-954)."""
    a, b = alpha.copy(), beta.copy()
    cs = np.zeros((len(a), 2))
    for i in range(len(a) - 1):
        r, c, s = drotg(a[i], b[i])
        a[i] = r
        cs[i] = (c, s)
        b[i] = s * a[i + 1]
        a[i + 1] = c * a[i + 1]
    return a, b, cs


def apply_house(house, tau, C):
    """dormqr('L','N'): C <- H_0 H_1 ... H_{m-1} C with reflector j stored in
    column j of ``house`` (unit diagonal)."""
    m = house.shape[0]
    C = C.copy()
    for j in range(m - 1, -1, -1):
        if tau[j] == 0.0:
            continue
        v = house[j:, j].copy()
        v[0] = 1.0
        C[j:] -= tau[j] * np.outer(v, v @ C[j:])
    return C


def leading_svd(a, b, k):
    """svd_mode 0: LAPACK SVD of the leading k x k bidiagonal (the reference
    calls dbdsdc with n = k, client.cpp:975-980); U m x k and V k x m padded
    with zeros as in the reference's zero-initialised buffers."""
    m = len(a)
    B = np.diag(a[:k]) + (np.diag(b[:k - 1], 1) if k > 1 else 0)
    Uk, s, Vk = np.linalg.svd(np.atleast_2d(B))
    U = np.zeros((m, k))
    V = np.zeros((k, m))
    U[:k] = Uk
    V[:, :k] = Vk
    return s, U, V


def _bsvd(alpha, beta, top_k, svd_mode):
    """lower -> upper, sigma count, the bidiagonal SVD and the sign convention
    (client.cpp:947-995); shared by both branches."""
    a, b, cs = lower_to_upper(alpha, beta)                        # :947-954
    bound = np.linalg.norm(a) ** 2 + np.linalg.norm(b) ** 2       # :966-971
    k = negative_count(a, b, bound) - negative_count(a, b, 0.0)
    if top_k > 0:
        k = min(k, top_k)
    if svd_mode in (0, 4):
        sigma, Ub, Vb = leading_svd(a, b, k)                      # :975-980 (dbdsdc)
    else:
        sigma, Ub, Vb = bidiagonal_svd(a, b, k)                   # :984
    for i in range(k):                                            # :988-995
        p = int(np.argmax(np.abs(Ub[:, i])))
        if Ub[p, i] < 0:
            Ub[:, i] = -Ub[:, i]
            Vb[i] = -Vb[i]
    return (a, b, cs), sigma, Ub, Vb, k


def _rotate_house(Ub, cs, house, tau):
    """U2 = H (G^T U_b): the Givens sweep undone, then the Ralha reflectors
    (client.cpp:1127-1128, 1135 / 1176)."""
    n = Ub.shape[0]
    U2 = Ub.copy()
    for i in range(n - 2, -1, -1):
        c_, s_ = cs[i]
        x, y = U2[i].copy(), U2[i + 1].copy()
        U2[i] = c_ * x - s_ * y
        U2[i + 1] = c_ * y + s_ * x
    return apply_house(house, tau, U2)


def run_tall(blocks_t, public_seed, private_seeds, top_k=-1, svd_mode=1, y=None, return_stages=False):
    """The tall-and-skinny branch, m > global_n (client.cpp:543-568, 627-679,
    805-814, 1002-1015, 1071-1105, 1119-1169).  The reference stores each
    participant's block transposed here: blocks_t[c] is X_c^T, local_n x m
    row-major (client.cpp:549, 1248).  Returns (sigma, FinalU k x m,
    [FinalVT_c k x local_n]); with svd_mode 4 (linear regression, labels y
    of length m) the third item is [w_c (local_n)] and FinalU is None."""
    P = len(blocks_t)
    m = blocks_t[0].shape[1]
    local_n = [x.shape[0] for x in blocks_t]
    global_n = sum(local_n)
    if m <= global_n:
        raise ValueError("run_tall needs m > global_n")
    stages = {}
    masked = []
    for c in range(P):                                            # :548-551
        x = np.ascontiguousarray(blocks_t[c], dtype=np.float64)
        x = block_shift_mask(x, MASK_PASSES, True, True, private_seeds[c])
        x = block_shift_mask(x, MASK_PASSES, True, False, public_seed)
        masked.append(x)
    Mt = np.concatenate(masked, axis=0)                           # global_n x m, repartition :627-659
    part, pos = row_split(m, P)
    npos = np.concatenate([[0], np.cumsum(local_n)])
    slabs, uq = [], []
    for c in range(P):
        S = Mt[:, pos[c]:pos[c + 1]].copy()                       # global_n x m_part
        if part[c] > global_n:                                    # :661-667
            r, q = local_qr(S)                                    # QR of S^T: R^T, Q^T (global_n x m_part)
            slabs.append(r)
            uq.append(q)
        else:
            slabs.append(S)
            uq.append(None)
    alpha, beta, house, tau, Vr = ralha(slabs)                    # bidiagonal_m = global_n, :805-910
    stages["ralha_lower"] = (alpha.copy(), beta.copy())
    (a, b, cs), sigma, Ub, Vb, k = _bsvd(alpha, beta, top_k, svd_mode)
    stages["bidiagonal"] = (a, b)
    compute_u, compute_v = svd_mode != 3, svd_mode != 2
    parts, FinalU, out3, sut = [], None, None, None
    if compute_u:                                                 # :1002-1015
        for c in range(P):
            t = Vb @ Vr[c]
            parts.append(t @ uq[c] if uq[c] is not None else t)  # k x m_part
        if svd_mode == 4:                                         # :1023-1044
            ym = block_shift_mask(np.asarray(y, float).reshape(1, m), MASK_PASSES, True, False, public_seed).ravel()
            sut = sum(parts[c] @ ym[pos[c]:pos[c + 1]] for c in range(P)) / sigma
        else:
            FinalU = np.concatenate(parts, axis=1)                # k x m, :1071-1096
            FinalU = block_shift_mask(FinalU, MASK_PASSES, False, False, public_seed)   # :1098-1105
    if compute_v:                                                 # :1119-1169
        U2 = _rotate_house(Ub, cs, house, tau)                    # global_n x k
        out3 = []
        if svd_mode == 4:
            w = U2 @ sut
            for c in range(P):
                wc = w[npos[c]:npos[c + 1]].reshape(1, -1)
                out3.append(block_shift_mask(wc, MASK_PASSES, False, False, private_seeds[c]).ravel())
        else:
            for c in range(P):
                t = np.ascontiguousarray(U2[npos[c]:npos[c + 1]].T)
                out3.append(block_shift_mask(t, MASK_PASSES, False, False, private_seeds[c]))
    out = (sigma, FinalU, out3)
    return (out + (stages,)) if return_stages else out


def run(blocks, public_seed, private_seeds, top_k=-1, svd_mode=1, return_stages=False):
    """DecentralizedClient::run(), opt_control 3, short-and-wide layout
    (m <= global_n, blocks X_c row-major m x local_n); svd_mode 0 (full,
    dbdsdc), 1 (two-sided), 2 (left only) or 3 (right only).  m == global_n
    runs without the global QR (client.cpp:795-798) and takes the V
    back-transform of the tall branch (:1129-1160)."""
    P = len(blocks)
    m = blocks[0].shape[0]
    local_n = [b.shape[1] for b in blocks]
    global_n = sum(local_n)
    if m > global_n:
        raise ValueError("m > global_n: the tall-and-skinny branch takes transposed blocks (run_tall)")
    if svd_mode == 4:
        raise ValueError("svd_mode 4 exists only in the tall-and-skinny branch (client.cpp:1180)")
    red = [reduced_width(m, n) for n in local_n]
    rg = sum(red)
    if rg <= m and m < global_n:
        raise ValueError("the V back-transform needs reduced_global_n > m (client.cpp:1179)")
    stages = {}
    masked, local_q = [], []
    for c in range(P):                                            # client.cpp:572-605
        x = np.ascontiguousarray(blocks[c], dtype=np.float64)
        if m < local_n[c] and (local_n[c] // m) > LOCAL_QR_THRESHOLD:
            r, q = local_qr(x)
        else:
            r, q = x.copy(), None
        stages.setdefault("local_r", []).append(r.copy())
        r = block_shift_mask(r, MASK_PASSES, True, True, public_seed)
        r = block_shift_mask(r, MASK_PASSES, True, False, private_seeds[c])
        masked.append(r)
        local_q.append(q)
    stages["masked"] = [x.copy() for x in masked]
    M = np.concatenate(masked, axis=1)                            # m x rg, repartition :681-703
    part, pos = row_split(m, P)
    Qg = None
    if rg > m:
        # global Householder QR of M^T (client.cpp:705-794), panel by panel in
        # the reference; one dgeqrf here (same reflectors, up to rounding)
        qr, tau_g, _, info = lapack.dgeqrf(np.asfortranarray(M.T))
        assert info == 0
        W = np.triu(qr[:m, :])
        Qg, _, info = lapack.dorgqr(qr, tau_g)
        assert info == 0
    else:
        W = M.T.copy()                                            # in-place transpose, :795-798
    stages["global_r"] = W.copy()
    slabs = [W[:, pos[c]:pos[c + 1]].copy() for c in range(P)]
    alpha, beta, house, tau, Vr = ralha(slabs)                    # :801-945
    stages["ralha_lower"] = (alpha.copy(), beta.copy())
    (a, b, cs), sigma, Ub, Vb, k = _bsvd(alpha, beta, top_k, svd_mode)
    stages["bidiagonal"] = (a.copy(), b.copy())
    stages["bsvd"] = (sigma.copy(), Ub.copy(), Vb.copy())
    FinalU = None
    if svd_mode != 3:                                             # :1002-1115
        FinalU = np.zeros((m, k))
        for c in range(P):
            FinalU[pos[c]:pos[c + 1]] = (Vb @ Vr[c]).T
        FinalU = block_shift_mask(FinalU, MASK_PASSES, False, True, public_seed)
    if svd_mode == 2:
        out = (sigma, FinalU, None)
        return (out + (stages,)) if return_stages else out
    U2 = _rotate_house(Ub, cs, house, tau)                        # :1127-1176
    FinalVT = []
    if m == global_n:                                             # :1129-1160
        npos = np.concatenate([[0], np.cumsum(local_n)])
        for c in range(P):
            t = np.ascontiguousarray(U2[npos[c]:npos[c + 1]].T)
            FinalVT.append(block_shift_mask(t, MASK_PASSES, False, False, private_seeds[c]))
    else:
        rpos = np.concatenate([[0], np.cumsum(red)])
        for c in range(P):
            t = U2.T @ Qg[rpos[c]:rpos[c + 1], :].T               # :1179
            t = block_shift_mask(t, MASK_PASSES, False, False, private_seeds[c])
            FinalVT.append(t @ local_q[c] if local_q[c] is not None else t)   # :1188-1195
    out = (sigma, FinalU, FinalVT)
    return (out + (stages,)) if return_stages else out
