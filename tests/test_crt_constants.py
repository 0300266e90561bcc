"""The arithmetic the CRT kernels (excalibur_b200/csrc/crt.cu) rely on,
checked on the CPU from the same moduli list and the same formulas for their
constants: the moduli are pairwise coprime bytes, the multiply-high
quotients are exact over the ranges the kernels feed them, the residues of
53-bit integers formed from the bytes of their offset FP64 bit patterns are
exact and stay in range, the epilogue's
reduction of an int32 accumulator is the residue, the modulus count covers
every product, and the fixed-point reconstruction recovers the integer."""
import math
import os
import re

import numpy as np
import pytest

SRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "excalibur_b200", "csrc", "crt.cu")


def moduli():
    text = open(SRC).read()
    body = re.search(r"MODULI\[MAXMOD\]\s*=\s*\{([^}]*)\}", text).group(1)
    return [int(v) for v in body.replace("\n", " ").split(",") if v.strip()]


MOD = moduli()


def crt_moduli(bits_a, bits_b, K):
    """crt.cu's rule: the fewest moduli (at least 4) whose product holds
    (bits_a - 2) + (bits_b - 2) + log2 K + 2 bits."""
    need = (bits_a - 2) + (bits_b - 2) + math.log2(max(K, 1)) + 2.0
    bits = 0.0
    for n, p in enumerate(MOD):
        bits += math.log2(p)
        if bits >= need:
            return max(n + 1, 4)
    return -1


def test_moduli_are_pairwise_coprime_bytes():
    assert len(MOD) == 24 and MOD[0] == 256
    assert all(2 <= p <= 256 for p in MOD)
    for i, p in enumerate(MOD):
        for q in MOD[i + 1:]:
            assert math.gcd(p, q) == 1, (p, q)


@pytest.mark.parametrize("p", MOD)
def test_multiply_high_quotients_are_exact(p):
    # magic32 = ceil(2^32 / p): exact quotients for 0 <= x < 2^24 (exhaustive)
    magic32 = -(-(1 << 32) // p)
    x = np.arange(1 << 24, dtype=np.uint64)
    assert np.array_equal((x * np.uint64(magic32)) >> np.uint64(32), x // np.uint64(p))


def dp4a(a, b, c):
    """Unsigned byte dot product of two 32-bit words plus c."""
    return c + sum(((a >> (8 * j)) & 255) * ((b >> (8 * j)) & 255) for j in range(4))


@pytest.mark.parametrize("p", MOD)
def test_residues_from_offset_bytes(p):
    """residues_rows/cols: t (an integer, |t| <= 2^51) + 1.5 2^52 is exact in
    FP64; its low word and its high word less 0x43300000 are the two words
    of u = t + 2^51 (also at t = 2^51, where y = 2^53); x = dp4a(lo, W0,
    dp4a(hi, W1, off)) with the byte weights 256^j mod p and off = -2^51 mod
    p in [1, p] lies in (0, 2^19) and is t mod p; the multiply-high quotient
    by ceil(2^32 / p) then gives the residue."""
    w = [(1 << (8 * j)) % p for j in range(7)]
    W0 = w[0] | w[1] << 8 | w[2] << 16 | w[3] << 24
    W1 = w[4] | w[5] << 8 | w[6] << 16
    off = p - (1 << 51) % p
    magic32 = -(-(1 << 32) // p)
    assert 1 <= off <= p
    rng = np.random.default_rng(p + 1)
    ts = [-(1 << 51), (1 << 51), (1 << 51) - 1, -(1 << 51) + 1, 0, -1, 1,
          *[int(v) for v in rng.integers(-(1 << 51), 1 << 51, 3000)]]
    y = np.array(ts, dtype=np.float64) + np.float64(1.5 * 2.0 ** 52)
    bits = y.view(np.uint64)
    for t, b in zip(ts, bits):
        lo, hi = int(b) & 0xFFFFFFFF, ((int(b) >> 32) - 0x43300000) & 0xFFFFFFFF
        u = t + (1 << 51)
        assert lo == u & 0xFFFFFFFF and hi == u >> 32 and hi <= 1 << 20
        x = dp4a(lo, W0, dp4a(hi, W1, off))
        assert 0 < x < (1 << 19)
        assert x - ((x * magic32) >> 32) * p == t % p


@pytest.mark.parametrize("p", MOD)
def test_epilogue_reduction_of_int32_accumulators(p):
    """The GEMM epilogue: an accumulator of at most 2^15 products of bytes in
    [0, 256) is 0 <= v < 2^31; x = (v >> 16) c16 + (v & 0xFFFF) < 2^24 and
    r = x - floor(x ceil(2^32 / p) / 2^32) p = v mod p."""
    c16, magic = 65536 % p, -(-(1 << 32) // p)
    top = (1 << 15) * 255 * 255
    assert top < (1 << 31)
    rng = np.random.default_rng(p + 2)
    vals = [0, 1, p - 1, p, (1 << 16) - 1, 1 << 16, top, *[int(v) for v in rng.integers(0, top + 1, 5000)]]
    for v in vals:
        x = (v >> 16) * c16 + (v & 0xFFFF)
        assert x < (1 << 24)
        r = x - ((x * magic) >> 32) * p
        assert r == v % p


@pytest.mark.parametrize("p", MOD)
def test_fused_epilogue_reduction(p):
    """The fused product's epilogue: the accumulator of u8 x u8 products over
    at most 2^15 terms is 0 <= v < 2^31, x = (v >> 16) c16 + (v & 0xFFFF) <
    2^24, r = x - floor(x ceil(2^32 / p) / 2^32) p = v mod p: the residue the
    two-pass path stores, which both paths then multiply by the same G limbs,
    so their outputs agree bit for bit."""
    c16, magic = 65536 % p, -(-(1 << 32) // p)
    rng = np.random.default_rng(p + 3)
    top = (1 << 15) * 255 * 255
    vals = [0, 1, p - 1, p, (1 << 16) - 1, 1 << 16, top, *[int(v) for v in rng.integers(0, top + 1, 5000)]]
    for v in vals:
        x = (v >> 16) * c16 + (v & 0xFFFF)
        assert x < (1 << 24)
        r = x - ((x * magic) >> 32) * p
        assert r == v % p


@pytest.mark.parametrize("bits_a,bits_b,K,expect", [(53, 53, 500_000, 16), (50, 50, 500_000, 15),
                                                    (53, 80, 1000, 19), (53, 80, 512, 18), (53, 53, 2000, 15)])
def test_modulus_count_covers_the_product(bits_a, bits_b, K, expect):
    n = crt_moduli(bits_a, bits_b, K)
    assert n == expect
    M = math.prod(MOD[:n])
    # |t| <= 2^(b-2) per operand, so |T| <= 2^(ba-2) 2^(bb-2) K <= M / 4
    assert 4 * (1 << (bits_a - 2)) * (1 << (bits_b - 2)) * K <= M


def glimbs(p, inv):
    """crt.cu's glimb_c: G = inv floor(2^128 / p) + floor(inv (2^128 mod p) / p)
    as four 32-bit limbs, least significant first."""
    F = (1 << 128) // p
    G = inv * F + (inv * ((1 << 128) % p)) // p
    return [(G >> (32 * l)) & 0xFFFFFFFF for l in range(4)]


def test_g_limbs_are_the_scaled_crt_digit():
    for n in (15, 16, 19, 24):
        M = math.prod(MOD[:n])
        for p in MOD[:n]:
            inv = pow((M // p) % p, -1, p)
            G = sum(v << (32 * l) for l, v in enumerate(glimbs(p, inv)))
            assert G == ((inv << 128) // p)


def reconstruct(T, n, limbs):
    """crt.cu's reconstruction: r_q = T mod p_q and the fraction S = sum_q r_q
    G_q mod 2^128, G_q = floor(2^128 ((M / p_q)^-1 mod p_q) / p_q) (its low 32
    bits dropped when limbs = 3), read as a signed 128-bit number: S M / 2^128
    is T up to the floors' errors."""
    ps = MOD[:n]
    M = math.prod(ps)
    S = 0
    for p in ps:
        inv = pow((M // p) % p, -1, p)
        G = sum(v << (32 * l) for l, v in enumerate(glimbs(p, inv)))
        if limbs == 3:
            G = (G >> 32) << 32
        S += (T % p) * G
    S %= 1 << 128
    if S >= 1 << 127:
        S -= 1 << 128
    return S, M


@pytest.mark.parametrize("n", [4, 15, 16, 19, 24])
@pytest.mark.parametrize("limbs", [3, 4])
def test_fixed_point_reconstruction(n, limbs):
    M = math.prod(MOD[:n])
    rng = np.random.default_rng(n * 10 + limbs)
    # the modulus count leaves M >= 4 max|T| (two bits of margin over the sign)
    Ts = [0, 1, -1, M // 4, -(M // 4)]
    Ts += [int(rng.integers(-(1 << 62), 1 << 62)) * int(rng.integers(1, 1 << 62)) % (M // 2) - M // 4
           for _ in range(300)]
    bits = 128 if limbs == 4 else 96
    for T in Ts:
        S, _ = reconstruct(T, n, limbs)
        # every term r_q G_q is short of r_q inv_q 2^128 / p_q by less than
        # r_q < 256 units of 2^(128 - bits): |S M - T 2^128| < n 256 M 2^(128 - bits)
        assert abs(S * M - T * (1 << 128)) < n * 256 * M * (1 << (128 - bits)), T
    # relative to the largest |T| the kernels allow (M / 4): below 2^-100 with
    # 128-bit fractions, 2^-70 with 96-bit ones
    assert n * 256 * 4 / float(1 << bits) < (2.0 ** -100 if limbs == 4 else 2.0 ** -70)
