"""The tall-and-skinny branch (m > global_n, client.cpp:543-568, 627-679,
805-814, 1002-1169), its linear-regression mode (svd_mode 4) and the
m == global_n case of the short-and-wide branch, on one GPU, against the
reference's own outputs (golden), the oracle and LAPACK."""
import numpy as np
import pytest

import cases
import oracle
from gpu_util import context, gap_groups, subspace_angle
from oracle import pipeline

pytestmark = pytest.mark.gpu
TALL = sorted(cases.tall_cases())
TALL_MODES = sorted(cases.tall_mode_cases())


@pytest.fixture(scope="module")
def ctx():
    return context()


def run(ctx, blocks, seed, precision=0, top_k=-1, svd_mode=1, y=None, tall=True):
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    dev = [ctx._dev(b.copy()) for b in blocks]
    lab = ctx._dev(y.copy()) if y is not None else None
    s, U, out3 = ctx.fedsvd(dev, pub, priv, top_k=top_k, svd_mode=svd_mode, precision=precision, tall=tall,
                            labels=lab)
    return (s.cpu().numpy(), None if U is None else U.cpu().numpy(),
            None if out3 is None else [v.cpu().numpy() for v in out3])


def check(g, s, U, out3, mode):
    assert len(s) == len(g["sigma"])
    assert np.max(np.abs(s - g["sigma"]) / g["sigma"]) < 1e-12
    if mode in (3, 4):
        assert U is None
    else:
        assert U.shape == g["U"].shape
        assert np.max(np.abs(U - g["U"])) < 1e-9
    if mode == 2:
        assert out3 is None
    elif mode == 4:
        for c, w in enumerate(out3):
            assert np.max(np.abs(w - g[f"w{c}"])) < 1e-10
    else:
        for c, v in enumerate(out3):
            assert np.max(np.abs(v - g[f"VT{c}"])) < 1e-9


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", TALL)
def test_tall_matches_reference(ctx, golden, name, precision):
    """FinalU (k x m) and every FinalVT_c of the reference's tall branch: slabs
    reduced by a local QR (t_qr), none reduced (t_noqr), only the first
    (t_mixed, m_part = 51, 50, 50 against global_n = 50)."""
    g = golden(f"pipe__{name}")
    blocks, seed, _ = cases.tall_cases()[name]
    check(g, *run(ctx, blocks, seed, precision), 1)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", TALL_MODES)
def test_tall_modes_match_reference(ctx, golden, name, precision):
    """svd_mode 0 (dbdsdc on the leading k x k bidiagonal), 2, 3, top-k and
    4 (linear regression: w_c in place of FinalVT_c)."""
    g = golden(f"pipe__{name}")
    case, mode, topk = cases.tall_mode_cases()[name]
    blocks, seed, y = cases.tall_cases()[case]
    check(g, *run(ctx, blocks, seed, precision, top_k=topk, svd_mode=mode, y=y if mode == 4 else None), mode)


@pytest.mark.parametrize("name", sorted(cases.square_cases()))
@pytest.mark.parametrize("mode", [0, 1])
def test_square_matches_reference(ctx, golden, mode, name):
    """m == global_n: no global QR, FinalVT_c from rows of the rotated U_b
    (client.cpp:795-798, 1129-1169); two participants and one."""
    g = golden(f"pipe__{name}_mode{mode}")
    blocks, seed = cases.square_cases()[name]
    for precision in (0, 1):
        check(g, *run(ctx, blocks, seed, precision, svd_mode=mode, tall=False), mode)


def test_tall_matches_oracle(ctx):
    blocks, seed, y = cases.tall_cases()["t_mixed"]
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    so, Uo, VTo = pipeline.run_tall(blocks, pub, priv)
    s, U, VT = run(ctx, blocks, seed)
    assert np.max(np.abs(s - so) / so) < 1e-12
    assert np.max(np.abs(U - Uo)) < 1e-9
    for v, vo in zip(VT, VTo):
        assert np.max(np.abs(v - vo)) < 1e-9


def test_tall_host_entry_equals_device_entry(ctx):
    blocks, seed, y = cases.tall_cases()["t_qr"]
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    s, U, VT = run(ctx, blocks, seed)
    s2, U2, VT2 = ctx.fedsvd_host(blocks, pub, priv, tall=True)
    assert np.array_equal(s, s2) and np.array_equal(U, U2)
    for a, b in zip(VT, VT2):
        assert np.array_equal(a, b)
    _, _, w = run(ctx, blocks, seed, svd_mode=4, y=y)
    _, U4, w2 = ctx.fedsvd_host(blocks, pub, priv, svd_mode=4, tall=True, labels=y)
    assert U4 is None
    for a, b in zip(w, w2):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", [0, 1])
def test_tall_large_against_lapack(ctx, precision):
    """P = 4, m = 40000 x global_n = 260 (every slab of 10000 rows reduced by a
    local QR, 3 GEMMs of the int8-slice kind in precision 1): singular values
    against LAPACK, subspaces, orthonormality, reconstruction, and the
    regression weights against a least-squares solve."""
    rng = np.random.default_rng(77)
    m, ln = 40000, (50, 70, 60, 80)
    A = rng.standard_normal((m, sum(ln))) @ np.diag(np.geomspace(1.0, 1e-3, sum(ln)))
    blocks, o = [], 0
    for n in ln:
        blocks.append(np.ascontiguousarray(A[:, o:o + n].T))
        o += n
    y = A @ rng.standard_normal(sum(ln)) + 1e-3 * rng.standard_normal(m)
    s, U, VT = run(ctx, blocks, 5, precision)
    Ul, sl, Vl = np.linalg.svd(A, full_matrices=False)
    assert np.max(np.abs(s - sl) / sl) < 1e-10
    assert np.max(np.abs(U @ U.T - np.eye(len(s)))) < 1e-11
    V = np.concatenate(VT, axis=1).T
    assert np.max(np.abs(V.T @ V - np.eye(len(s)))) < 1e-11
    assert np.max(np.abs(U.T @ np.diag(s) @ V.T - A)) < 1e-12 * np.abs(A).max() * 100
    for grp in gap_groups(sl):
        assert subspace_angle(U.T[:, grp], Ul[:, grp]) < 1e-8
        assert subspace_angle(V[:, grp], Vl[grp].T) < 1e-8
    _, _, w = run(ctx, blocks, 5, precision, svd_mode=4, y=y)
    wl = np.linalg.lstsq(A, y, rcond=None)[0]
    assert np.max(np.abs(np.concatenate(w) - wl)) / np.max(np.abs(wl)) < 1e-9


def test_lr_refused_short_and_wide(ctx):
    """The reference implements linear regression only for m > global_n
    (client.cpp:1180 asserts svd_mode != 4 on the other branch)."""
    blocks, seed = cases.pipeline_cases()["noqr"]
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    with pytest.raises(RuntimeError, match="svd_mode 4"):
        ctx.fedsvd([ctx._dev(b.copy()) for b in blocks], pub, priv, svd_mode=4,
                   labels=ctx._dev(np.ones(blocks[0].shape[0])))
