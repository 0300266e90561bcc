"""Pins the oracle (oracle/bbt_oracle.cpp, oracle/pipeline.py) against
golden vectors produced by the reference's own sources
(tests/golden/make_golden.py).  CPU only."""
import glob
import hashlib
import os

import numpy as np
import pytest

import cases
import oracle
from oracle import pipeline

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


BIDIAG = sorted(cases.bidiagonal_cases())
MASKS = sorted(cases.mask_cases())
PIPES = sorted(cases.pipeline_cases())


def test_every_fixture_has_a_case():
    names = {os.path.basename(f)[:-4] for f in glob.glob(os.path.join(GOLD, "*.npz"))}
    want = ({f"bidiag__{n}" for n in BIDIAG} | {f"mask__{n}" for n in MASKS}
            | {f"pipe__{n}" for n in PIPES} | {f"pipe__{n}" for n in cases.pipeline_mode_cases()}
            | {f"pipe__{n}" for n in cases.tall_cases()} | {f"pipe__{n}" for n in cases.tall_mode_cases()}
            | {f"pipe__{n}_mode{m}" for n in cases.square_cases() for m in (0, 1)}
            | {f"step__{n}" for n in cases.step_cases()} | {f"gen__{n}" for n in cases.GENERATOR_FIXTURES}
            | {f"omask__{n}" for n in cases.OTHER_MASK_CASES})
    assert names == want


@pytest.mark.parametrize("name", BIDIAG)
def test_sturm_counts_exact(golden, name):
    g = golden(f"bidiag__{name}")
    a, b = g["alpha"], g["beta"]
    got = [oracle.negative_count(a, b, mu) for mu in g["mus"]]
    assert np.array_equal(np.array(got, dtype=np.int32), g["counts"])


@pytest.mark.parametrize("name", BIDIAG)
def test_bidiagonal_svd(golden, name):
    g = golden(f"bidiag__{name}")
    top_k = int(g["top_k"])
    # singular values: bit-exact from the reference's own bisection bound
    # (same Sturm arithmetic, same bisection tree)
    s0 = oracle.bisection(g["alpha"], g["beta"], 0.0, float(g["bound"]), 1e-20, top_k)
    assert np.array_equal(s0, g["sigma"])
    s, U, V = oracle.bidiagonal_svd(g["alpha"], g["beta"], top_k)
    # with the oracle's own 2-norm in the bound: a leaf is independent of the
    # starting interval once it is two adjacent doubles, so values >= 1e-4
    # stay bit-exact; below that the 1e-20 absolute width test ends the
    # search first and the leaf may move by < 1e-20
    big = g["sigma"] >= 1e-4
    assert np.array_equal(s[big], g["sigma"][big])
    assert np.max(np.abs(s - g["sigma"]), initial=0.0) <= 2e-20
    # vectors: the reference normalises with BLAS dnrm2, the oracle with its
    # own scaled 2-norm, so they agree to a few ulps.  Where the qd
    # recurrences break down (clusters below the twisted method's reach) the
    # reference's vectors are NaN and which NaN cblas_idamin picks is up to
    # the BLAS build; only the reference's finite vectors are compared.
    ok_u = np.isfinite(g["U"]).all(axis=0)
    ok_v = np.isfinite(g["V"]).all(axis=1)
    assert np.max(np.abs(U - g["U"])[:, ok_u], initial=0.0) < 1e-13
    assert np.max(np.abs(V - g["V"])[ok_v], initial=0.0) < 1e-13
    if name != "cluster_k64":
        assert ok_u.all() and ok_v.all()


@pytest.mark.parametrize("name", MASKS)
def test_masks_bit_exact(golden, name):
    g = golden(f"mask__{name}")
    x, passes, mask, is_left, seed, fn = cases.mask_cases()[name]
    assert sha(x) == str(g["x_sha"])
    f = oracle.givens_mask if fn == "givens" else oracle.block_shift_mask
    y = f(x, passes, mask, is_left, seed)
    assert np.array_equal(y, g["y"])


@pytest.mark.parametrize("name", PIPES)
def test_pipeline_matches_reference(golden, name):
    g = golden(f"pipe__{name}")
    blocks, seed = cases.pipeline_cases()[name]
    assert sha(*blocks) == str(g["x_sha"])
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    s, U, VT = pipeline.run(blocks, pub, priv)
    assert len(s) == len(g["sigma"])
    assert np.max(np.abs(s - g["sigma"]) / g["sigma"]) < 1e-13
    assert np.max(np.abs(U - g["U"])) < 1e-10
    for c, v in enumerate(VT):
        assert np.max(np.abs(v - g[f"VT{c}"])) < 1e-10


def test_pipeline_against_lapack_svd():
    blocks, seed = cases.pipeline_cases()["c1"]
    pub, priv = oracle.reference_seeds(seed, 2)
    s, U, VT = pipeline.run(blocks, pub, priv)
    X = np.concatenate(blocks, axis=1)
    sv = np.linalg.svd(X, compute_uv=False)
    assert np.max(np.abs(s - sv) / sv) < 1e-12
    assert np.max(np.abs(U @ np.diag(s) @ np.concatenate(VT, axis=1) - X)) < 1e-11


MODES = sorted(cases.pipeline_mode_cases())


@pytest.mark.parametrize("name", MODES)
def test_pipeline_modes_match_reference(golden, name):
    g = golden(f"pipe__{name}")
    case, mode, topk = cases.pipeline_mode_cases()[name]
    blocks, seed = cases.pipeline_cases()[case]
    assert sha(*blocks) == str(g["x_sha"])
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    s, U, VT = pipeline.run(blocks, pub, priv, top_k=topk, svd_mode=mode)
    assert len(s) == len(g["sigma"])
    assert np.max(np.abs(s - g["sigma"]) / g["sigma"]) < 1e-13
    if mode != 3:
        assert np.max(np.abs(U - g["U"])) < 1e-10
    else:
        assert U is None and "U" not in g
    if mode != 2:
        for c, v in enumerate(VT):
            assert np.max(np.abs(v - g[f"VT{c}"])) < 1e-10
    else:
        assert VT is None


TALL = sorted(cases.tall_cases())
TALL_MODES = sorted(cases.tall_mode_cases())


def _check_outputs(g, s, U, out3, mode):
    assert len(s) == len(g["sigma"])
    assert np.max(np.abs(s - g["sigma"]) / g["sigma"]) < 1e-13
    if mode not in (3, 4):
        assert np.max(np.abs(U - g["U"])) < 1e-10
    else:
        assert U is None and "U" not in g
    if mode == 4:
        for c, w in enumerate(out3):
            assert np.max(np.abs(w - g[f"w{c}"])) < 1e-12
    elif mode != 2:
        for c, v in enumerate(out3):
            assert np.max(np.abs(v - g[f"VT{c}"])) < 1e-10
    else:
        assert out3 is None


@pytest.mark.parametrize("name", TALL)
def test_tall_pipeline_matches_reference(golden, name):
    g = golden(f"pipe__{name}")
    blocks, seed, _ = cases.tall_cases()[name]
    assert sha(*blocks) == str(g["x_sha"])
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    s, U, VT, st = pipeline.run_tall(blocks, pub, priv, return_stages=True)
    _check_outputs(g, s, U, VT, 1)
    a, b = st["bidiagonal"]
    assert np.max(np.abs(np.abs(np.concatenate([a, b])) - np.abs(g["ab"]))) < 1e-10


@pytest.mark.parametrize("name", TALL_MODES)
def test_tall_modes_match_reference(golden, name):
    g = golden(f"pipe__{name}")
    case, mode, topk = cases.tall_mode_cases()[name]
    blocks, seed, y = cases.tall_cases()[case]
    assert sha(*blocks, y) == str(g["x_sha"])
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    s, U, out3 = pipeline.run_tall(blocks, pub, priv, top_k=topk, svd_mode=mode, y=y)
    _check_outputs(g, s, U, out3, mode)


def test_tall_lr_is_least_squares():
    """svd_mode 4 returns w = V diag(1/sigma) U^T y, the least-squares solution
    of X w = y with X = [X_0 | X_1 | ...] (client.cpp:1023-1160)."""
    blocks, seed, y = cases.tall_cases()["t_qr"]
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    _, _, w = pipeline.run_tall(blocks, pub, priv, svd_mode=4, y=y)
    X = np.concatenate([b.T for b in blocks], axis=1)
    assert np.max(np.abs(np.concatenate(w) - np.linalg.lstsq(X, y, rcond=None)[0])) < 1e-12


@pytest.mark.parametrize("name", sorted(cases.square_cases()))
@pytest.mark.parametrize("mode", [0, 1])
def test_square_matches_reference(golden, mode, name):
    g = golden(f"pipe__{name}_mode{mode}")
    blocks, seed = cases.square_cases()[name]
    assert sha(*blocks) == str(g["x_sha"])
    pub, priv = oracle.reference_seeds(seed, len(blocks))
    s, U, VT = pipeline.run(blocks, pub, priv, svd_mode=mode)
    _check_outputs(g, s, U, VT, mode)


@pytest.mark.parametrize("name", sorted(n for n, c in cases.OTHER_MASK_CASES.items() if c[0] in ("naive", "cached")))
def test_givens_variants_match_reference(golden, name):
    """The oracle's restatement of naive_givens_mask_parallel and
    givens_mask_cache_optimized_parallel against the reference's build: the
    cache-optimised mask to the last bit, the naive one to rounding (the
    reference rotates with its BLAS drot); glibc's rand() state afterwards
    exactly."""
    key, m, n, passes, _, mask, left, seed = cases.OTHER_MASK_CASES[name]
    g = golden(f"omask__{name}")
    y = oracle.givens_variant(g["x_in"].reshape(m, n), passes, mask, left, seed, key == "cached").reshape(-1)
    if key == "cached":
        assert np.array_equal(y, g["x_out"])
    else:
        assert np.abs(y - g["x_out"]).max() <= 1e-14 * np.abs(g["x_out"]).max()
    assert oracle.rand() == int(g["rand_after"])


@pytest.fixture(scope="module")
def lapack():
    import ctypes
    import site
    hits = [h for d in site.getsitepackages() for h in glob.glob(os.path.join(d, "scipy.libs", "libscipy_openblas-*.so"))]
    if not hits:
        pytest.skip("no LAPACK library in this environment")
    ctypes.CDLL(hits[0], mode=ctypes.RTLD_GLOBAL)   # found by the oracle at run time


@pytest.mark.parametrize("name", sorted(n for n, c in cases.OTHER_MASK_CASES.items() if c[0] not in ("naive", "cached")))
def test_dense_masks_match_reference(golden, lapack, name):
    """The oracle's restatement of block_mask, shuffle_block_mask, house_mask
    and householder_reflector_mask (reflectors applied one by one, as
    dormqr defines them) against the reference's build, to rounding; glibc's
    rand() state afterwards exactly."""
    key, m, n, size, rounds, mask, left, seed = cases.OTHER_MASK_CASES[name]
    g = golden(f"omask__{name}")
    y = oracle.dense_mask(key, g["x_in"].reshape(m, n), size, mask, left, seed, rounds).reshape(-1)
    assert np.abs(y - g["x_out"]).max() <= 1e-13 * np.abs(g["x_out"]).max()
    assert oracle.rand() == int(g["rand_after"])


@pytest.mark.parametrize("name", sorted(cases.step_cases()))
def test_oracle_steps_match_reference(golden, name):
    """The per-step helpers (bbtsvd.cpp:54-164, 970-978) restated in
    oracle/steps.py against the reference's own outputs: the qd recurrences,
    the Householder vector and the rotation bit for bit, the normalised
    inverse-iteration vector to rounding (the reference's dnrm2)."""
    from oracle import steps
    g = golden(f"step__{name}")
    a, b = list(g["alpha"]), list(g["beta"])
    l, d = steps.ldl_decomposition(a, b)
    assert np.array_equal(l, g["l"]) and np.array_equal(d, g["d"])
    tau = float(g["omega"]) ** 2
    lp, dp, s = steps.dstqds(l, d, tau)
    assert np.array_equal(lp, g["lp"]) and np.array_equal(dp, g["dp"]) and np.array_equal(s, g["s"])
    up, rp, p = steps.dpqds(l, d, tau)
    assert np.array_equal(up, g["up"]) and np.array_equal(rp, g["rp"]) and np.array_equal(p, g["p"])
    n = len(a)
    v = steps.inverse_iteration(n, int(g["twist"]), lp, up)
    assert np.max(np.abs(np.array(v) - g["vi"][::2])) < 1e-15
    inc = int(g["house_inc"])
    hx, beta = steps.generate_house(list(g["house_in"][::inc]))
    out = g["house_in"].copy()
    out[::inc] = hx
    assert np.array_equal(out, g["house_out"]) and beta == float(g["house_beta"][0])
    x, y = steps.mmap_drot(a, list(np.resize(g["beta"], n)), float(g["drot_c"]), float(g["drot_s"]))
    assert np.array_equal(x, g["drot_x"]) and np.array_equal(y, g["drot_y"])
