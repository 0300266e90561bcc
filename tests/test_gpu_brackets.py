"""Learned bisection brackets: the library's MLP kernels against the numpy
restatement (forward, loss, gradient, features), training on the GPU, and the
bracketed bisection -- bit-identical to the plain bisection whatever the
brackets (perfect, garbage or learned), with fewer Sturm evaluations when the
learned brackets are good."""
import os

import numpy as np
import pytest

import cases
from gpu_util import context
from oracle import mlp

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return context()


def test_forward_matches_numpy(ctx):
    rng = np.random.default_rng(0)
    theta = mlp.init(2) + 0.05 * rng.standard_normal(mlp.NPARAM)
    X = rng.standard_normal((1000, mlp.F))
    assert ctx.mlp_param_count() == mlp.NPARAM
    out = ctx.mlp_forward(X, theta).cpu().numpy()
    ref, _ = mlp.forward(theta, X)
    assert np.max(np.abs(out - ref)) < 1e-12 * max(1.0, np.max(np.abs(ref)))


def test_gradient_matches_numpy(ctx):
    rng = np.random.default_rng(1)
    theta = mlp.init(3) + 0.05 * rng.standard_normal(mlp.NPARAM)
    X = rng.standard_normal((777, mlp.F)) * 0.5
    y = rng.uniform(-40, 0, 777) / 8.0
    g, loss = ctx.mlp_grad(X, y, theta)
    lref, gref = mlp.loss_grad(theta, X, y)
    assert abs(float(loss) - lref) <= 1e-12 * abs(lref)
    g = g.cpu().numpy()
    assert np.max(np.abs(g - gref)) <= 1e-11 * np.max(np.abs(gref))


@pytest.mark.parametrize("name", ["rand_k100", "graded_signed_k64", "cluster_k64"])
def test_features_match_numpy(ctx, name):
    a, b, _ = cases.bidiagonal_cases()[name]
    X = ctx.mlp_features(a, b).cpu().numpy()
    ref, _ = mlp.features(a, b)
    assert np.max(np.abs(X - ref)) < 1e-14


def plain_and_bracketed(ctx, a, b, br):
    s0 = ctx.bidiagonal_singular_values(a, b)
    s1, st = ctx.bidiagonal_singular_values(a, b, brackets=br)
    return s0.cpu().numpy(), s1.cpu().numpy(), st


def plain_evals(ctx, a, b):
    k = len(a)
    br = np.tile([1.0, 0.5], (k, 1))     # empty brackets: never a candidate, no jump
    s0, s1, st = plain_and_bracketed(ctx, a, b, br)
    assert np.array_equal(s0, s1) and st["jumps"] == 0 and st["verify_evals"] == 0
    return st["sturm_evals"]


@pytest.mark.parametrize("name", sorted(cases.bidiagonal_cases()))
def test_bracketed_bisection_bit_identical(ctx, name):
    """Perfect, garbage and random brackets: the same singular values as the
    plain bisection, bit for bit (verification rejects what is wrong)."""
    a, b, _ = cases.bidiagonal_cases()[name]
    s0 = ctx.bidiagonal_singular_values(a, b).cpu().numpy()
    k = len(s0)
    if k == 0:
        return
    rng = np.random.default_rng(k)
    perfect = np.stack([s0 * (1 - 1e-13), s0 * (1 + 1e-13)], axis=1)
    garbage = np.sort(rng.uniform(0, 2 * s0.max(), (k, 2)), axis=1)
    shifted = np.stack([s0 * 1.5, s0 * 2.0], axis=1)            # every bracket misses its value
    for br in (perfect, garbage, shifted):
        _, s1, st = plain_and_bracketed(ctx, a, b, br)
        assert np.array_equal(s0, s1), st
    _, _, st = plain_and_bracketed(ctx, a, b, perfect)
    assert st["jumps"] >= 1 or k == 1


def test_perfect_brackets_save_sturm_counts(ctx):
    rng = np.random.default_rng(8)
    k = 400
    a, b = rng.uniform(0.5, 2.0, k), rng.uniform(-1, 1, k - 1)
    s0 = ctx.bidiagonal_singular_values(a, b).cpu().numpy()
    base = plain_evals(ctx, a, b)
    perfect = np.stack([s0 * (1 - 1e-12), s0 * (1 + 1e-12)], axis=1)
    _, s1, st = plain_and_bracketed(ctx, a, b, perfect)
    assert np.array_equal(s0, s1)
    assert st["jumps"] > k // 2 and st["verify_evals"] == 2 * st["jumps"]
    assert st["sturm_evals"] < 0.75 * base, (st, base)


def test_training_reduces_loss(ctx):
    """The device training loop (gradient + Adam kernels) fits a small set of
    method-generated bidiagonals."""
    from excalibur_b200 import brackets
    X, y = brackets.build_dataset(ctx, 12, [128, 192], ["geometric", "clustered"], seed=77)
    theta, hist = brackets.fit(ctx, X, y, steps=400, batch=1024, lr=3e-3, seed=1)
    assert hist[-1][1] < hist[0][1] - 1.0, hist[:3] + hist[-3:]
    # the GPU loss agrees with the numpy loss of the trained parameters
    lref, _ = mlp.loss_grad(theta, X.cpu().numpy(), y.cpu().numpy())
    _, loss = ctx.mlp_grad(X, y, theta)
    assert abs(float(loss) - lref) <= 1e-10 * max(1.0, abs(lref))


MODEL = os.path.join(os.path.dirname(__file__), "..", "excalibur_b200", "data", "bracket_mlp.npz")


@pytest.mark.parametrize("family", ["geometric", "clustered"])
def test_trained_model_gain(ctx, family):
    """What the committed model gains over the plain bisection on fresh
    bidiagonals of its training families (seeds outside the training set):
    the singular values are identical, and the Sturm evaluations are never
    more than 1% above the plain count (verification is lazy, so brackets too
    wide to skip a level cost nothing).  The measured gain is printed; on
    these families it is ~0 because the model's log-spread (~0.16 octave) is
    wider than the gaps between neighbouring values (0.016 octave for the
    geometric family, 1e-10 relative inside clusters), and a bracket can only
    skip the levels below the one where bisection isolates its value."""
    from excalibur_b200 import brackets
    theta, z = brackets.load_model(MODEL)
    gains = []
    for seed in (901, 902):
        a, b = brackets.make_bidiagonal(ctx, family, 1024, seed)
        a, b = a.cpu().numpy(), b.cpu().numpy()
        base = plain_evals(ctx, a, b)
        for zz in (1.0, 2.0, z):
            br = ctx.mlp_brackets(a, b, theta, z=zz)
            s0, s1, st = plain_and_bracketed(ctx, a, b, br)
            assert np.array_equal(s0, s1)
            print(f"{family} seed {seed} z {zz}: plain {base} evals, learned {st['sturm_evals']} "
                  f"(jumps {st['jumps']}, verification {st['verify_evals']} evals, rounds {st['rounds']}), "
                  f"gain {1.0 - st['sturm_evals'] / base:.3f}")
            gains.append(1.0 - st["sturm_evals"] / base)
    assert min(gains) > -0.01, gains


def test_bracket_model_inside_pipeline(ctx):
    """set_bracket_model: the dense SVD returns the same singular values with
    the model on (the brackets only ever skip levels)."""
    from excalibur_b200 import brackets
    theta, z = brackets.load_model(MODEL)
    rng = np.random.default_rng(5)
    m = 256
    sv = np.geomspace(1.0, 1e-5, m)
    q1, _ = np.linalg.qr(rng.standard_normal((m, m)))
    q2, _ = np.linalg.qr(rng.standard_normal((m, m)))
    X = (q1 * sv) @ q2.T
    s0 = ctx.svd_dense(ctx._dev(X.copy()))[0].cpu().numpy()
    ctx.set_bracket_model(theta, z)
    try:
        s1 = ctx.svd_dense(ctx._dev(X.copy()))[0].cpu().numpy()
        st = ctx.bisection_stats()
    finally:
        ctx.set_bracket_model(None)
    assert np.array_equal(s0, s1)
    assert st["rounds"] > 0, st
