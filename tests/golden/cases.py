"""Seeded inputs of the golden fixtures (shared by make_golden.py and the
tests).  Shapes follow the reference's own conventions: a participant's block
is row-major m x local_n (Excalibur client.hpp:39-44, generate_data.cpp)."""
import numpy as np


def bidiagonal_cases():
    """name -> (alpha, beta, top_k)."""
    out = {}
    rng = np.random.default_rng(20240601)
    for k in (1, 2, 3, 5, 31, 33, 100, 257):
        a = rng.uniform(0.5, 2.0, k)
        b = rng.uniform(-1.0, 1.0, k - 1)
        out[f"rand_k{k}"] = (a, b, k)
    a = rng.uniform(0.5, 2.0, 100)
    b = rng.uniform(-1.0, 1.0, 99)
    out["topk_k100_t10"] = (a, b, 10)
    k = 64
    a = np.geomspace(1.0, 1e-6, k) * rng.choice([-1.0, 1.0], k)
    b = 0.3 * np.geomspace(1.0, 1e-6, k)[1:] * rng.choice([-1.0, 1.0], k - 1)
    out["graded_signed_k64"] = (a, b, k)
    centres = np.geomspace(1.0, 1e-3, 4)
    a = np.concatenate([c * (1.0 + 1e-10 * np.arange(16)) for c in centres])
    b = 1e-13 * rng.uniform(-1.0, 1.0, 63)
    out["cluster_k64"] = (a, b, 64)
    return out


def sturm_shifts(a, b):
    k = len(a)
    B = np.diag(a) + (np.diag(b, 1) if k > 1 else 0)
    s = np.linalg.svd(np.atleast_2d(B), compute_uv=False)
    bound = np.linalg.norm(a) ** 2 + (np.linalg.norm(b) ** 2 if k > 1 else 0.0)
    rng = np.random.default_rng(k)
    mus = np.concatenate([[0.0, bound, s.max() * 1.5], s, rng.uniform(0, s.max(), 16)])
    return mus.astype(np.float64)


def mask_cases():
    """name -> (x, passes, mask, is_left, seed, fn)."""
    out = {}
    rng = np.random.default_rng(7)
    shapes = [
        ("sq100_left", (100, 100), 1, 1, 11, "givens"),
        ("sq100_right", (100, 100), 1, 0, 12, "givens"),
        ("sq100_left_unmask", (100, 100), 0, 1, 11, "givens"),
        ("wide_right", (37, 1000), 1, 0, 13, "givens"),
        ("tall_left", (1000, 37), 1, 1, 14, "givens"),
        ("odd_left", (33, 17), 1, 1, 15, "givens"),
        ("odd_right", (17, 33), 1, 0, 16, "givens"),
        ("odd_left_unmask", (33, 17), 0, 1, 15, "givens"),
        ("odd_right_unmask", (17, 33), 0, 0, 16, "givens"),
        ("k2_left", (2, 9), 1, 1, 17, "givens"),
        ("k3_right", (6, 3), 1, 0, 18, "givens"),
        ("tail_left", (5, 7), 1, 1, 19, "givens"),
        ("bsm_direct", (64, 48), 1, 1, 20, "block_shift"),
        ("bsm_virtual_rem", (1, 10007), 1, 0, 21, "block_shift"),
        ("bsm_virtual_rem_unmask", (1, 10007), 0, 0, 21, "block_shift"),
        ("bsm_virtual_exact", (2, 10240), 1, 0, 22, "block_shift"),
        ("bsm_virtual_left", (10009, 2), 1, 1, 23, "block_shift"),
    ]
    for name, shp, mask, left, seed, fn in shapes:
        out[name] = (rng.standard_normal(shp), 32, mask, left, seed, fn)
    return out


def pipeline_mode_cases():
    """name -> (pipeline case, svd_mode, top_k): the other svd modes and top-k
    on the same inputs (client.cpp:186-192, 971)."""
    return {"c1_mode0": ("c1", 0, -1), "c1_mode2_top10": ("c1", 2, 10), "c1_mode3_top10": ("c1", 3, 10),
            "c1_mode1_top10": ("c1", 1, 10), "p3_mode0_top7": ("p3_uneven", 0, 7)}


def pipeline_cases():
    """name -> (blocks, seed).  ``c1`` is the 2 x (1000 x 100) N(0,1) case
    (row-stacked 2000 x 100), held as the reference's m=100 x local_n=1000."""
    out = {}
    rng = np.random.default_rng(0)
    out["c1"] = ([rng.standard_normal((1000, 100)).T.copy() for _ in range(2)], 0)
    rng = np.random.default_rng(5)
    out["p3_uneven"] = ([rng.standard_normal((48, n)) for n in (400, 290, 150)], 5)
    rng = np.random.default_rng(9)
    out["noqr"] = ([rng.standard_normal((40, n)) for n in (160, 200)], 9)
    return out


def tall_cases():
    """name -> (blocks_t, seed, y): the tall-and-skinny branch (m > global_n),
    where the reference holds each participant's block transposed, local_n x m
    row-major (client.cpp:549, 1248); y (length m) is the label vector of
    svd_mode 4, held by the last participant (client.cpp:1026-1029)."""
    out = {}
    rng = np.random.default_rng(31)
    # every column slab m_part = 250 > global_n = 80: local QR of each slab
    out["t_qr"] = ([rng.standard_normal((n, 500)) for n in (30, 50)], 31, rng.standard_normal(500))
    rng = np.random.default_rng(32)
    # m_part = 34, 33, 33 <= global_n = 75: slabs go to Ralha as they are
    out["t_noqr"] = ([rng.standard_normal((n, 100)) for n in (20, 30, 25)], 32, rng.standard_normal(100))
    rng = np.random.default_rng(33)
    # m_part = 51, 50, 50 against global_n = 50: only the first slab is reduced
    out["t_mixed"] = ([rng.standard_normal((n, 151)) for n in (10, 25, 15)], 33, rng.standard_normal(151))
    rng = np.random.default_rng(34)
    # one participant, m = 120 > global_n = 30: a slab QR of its whole block
    out["t_p1"] = ([rng.standard_normal((30, 120))], 34, rng.standard_normal(120))
    return out


def tall_mode_cases():
    """name -> (tall case, svd_mode, top_k)."""
    return {"t_qr_mode0": ("t_qr", 0, -1), "t_qr_mode2_top10": ("t_qr", 2, 10),
            "t_qr_mode3_top10": ("t_qr", 3, 10), "t_qr_mode4": ("t_qr", 4, -1),
            "t_mixed_mode4": ("t_mixed", 4, -1), "t_noqr_mode1_top7": ("t_noqr", 1, 7)}


def square_cases():
    """name -> (blocks, seed): m == global_n in the short-and-wide layout, the
    case without a global QR whose V comes from rows of the rotated bidiagonal
    U (client.cpp:795-798, 1129-1160)."""
    rng = np.random.default_rng(41)
    out = {"sq80": ([rng.standard_normal((80, n)) for n in (30, 50)], 41)}
    # one participant (the reference's -t 1), square: the shape its single-process run supports
    rng = np.random.default_rng(10)
    out["sq60_p1"] = ([rng.standard_normal((60, 60))], 10)
    return out


def step_cases():
    """name -> (alpha, beta, omega index, twist index k, house x, house inc,
    drot (c, s)): inputs of the reference's per-step helpers
    (ldl_decomposition, dstqds, dpqds, inverse_iteration,
    one_pair_singular_vector_twisted_factorization, generate_house, mmap_drot,
    bbtsvd.cpp:54-164, 970-978), taken from the bidiagonal cases."""
    out = {}
    rng = np.random.default_rng(99)
    for name in ("rand_k100", "rand_k257", "graded_signed_k64", "rand_k5"):
        a, b, _ = bidiagonal_cases()[name]
        k = len(a)
        x = rng.standard_normal(3 * k)
        th = rng.uniform(0, 2 * np.pi)
        out[name] = (a, b, min(3, k - 1), k // 2, x, 3, (np.cos(th), np.sin(th)))
    a, b, _ = bidiagonal_cases()["rand_k31"]
    out["house_zero_tail_neg"] = (a, b, 0, 0, np.array([-2.0] + [0.0] * 9), 1, (0.6, 0.8))
    out["house_zero_tail_pos"] = (a, b, 0, 0, np.array([2.0] + [0.0] * 9), 1, (0.6, -0.8))
    return out


# Fixtures of the reference's random orthogonal matrix generators and
# shuffle_matrix (make_golden.py generator_fixtures): name -> its test.
GENERATOR_FIXTURES = ("house_row7", "house_col6", "orth_tall9x4", "orth_wide4x9", "shuffle_left7x5",
                      "unshuffle_left7x5", "shuffle_right6x9", "unshuffle_right6x9", "shuffle_left8x3")


# The other masks of bbtsvd.hpp (make_golden.py other_mask_fixtures): name ->
# (function, m, n, size, rounds, mask, is_left, seed); size is the pass count,
# block size or reflector count, rounds the shuffle_block_mask rounds.  The
# block masks' cases use one block smaller than the block size: a full block
# makes the reference read its tau array one past the end (bbtsvd.cpp:433,
# 441, 503), whose value is whatever the allocator left there.
OTHER_MASK_CASES = {
    "naive_left7x5": ("naive", 7, 5, 3, 0, 1, 1, 4),
    "naive_right6x9": ("naive", 6, 9, 2, 0, 0, 0, 13),
    "naive_left8x4": ("naive", 8, 4, 4, 0, 0, 1, 7),
    "cached_left7x5": ("cached", 7, 5, 3, 0, 1, 1, 4),
    "cached_right6x9": ("cached", 6, 9, 2, 0, 0, 0, 13),
    "cached_left5x8": ("cached", 5, 8, 3, 0, 0, 1, 21),
    "block_left7x5": ("block", 7, 5, 9, 0, 1, 1, 5),
    "block_right6x9": ("block", 6, 9, 12, 0, 0, 0, 6),
    "block_right8x6": ("block", 8, 6, 8, 0, 1, 0, 2),
    "shufblock_left7x5": ("shufblock", 7, 5, 8, 2, 1, 1, 8),
    "shufblock_right6x9": ("shufblock", 6, 9, 10, 2, 0, 0, 3),
    "house_left6x4": ("house", 6, 4, 3, 0, 1, 1, 10),
    "house_right5x7": ("house", 5, 7, 7, 0, 0, 0, 12),
    "reflector_left6x4": ("reflector", 6, 4, 3, 0, 1, 1, 14),
    "reflector_left4x7": ("reflector", 4, 7, 4, 0, 0, 1, 15),
    "reflector_right5x8": ("reflector", 5, 8, 5, 0, 1, 0, 16),
}
