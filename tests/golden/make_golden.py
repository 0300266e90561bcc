"""Generate the golden fixtures in tests/golden/ from the REFERENCE itself.

Runs the reference's own sources, compiled by ``make -C oracle ref`` from
the Excalibur checkout (default /root/reference; override with
EXCALIBUR_REF), never the oracle restatement:

* ``oracle/_ref/libref_capi.so``: the reference's bbtsvd.hpp functions
  (negative_count, bisection_singular_values,
  bidiagonal_bisection_twisted_svd, givens_mask_..._with_simd,
  block_shift_mask) called through extern "C" wrappers;
* ``oracle/_ref/ref_pipeline``: one reference participant
  (DecentralizedClient::run(), svd_mode 1, opt 3) per process over
  loopback TCP, P processes per case.

Inputs are regenerated from numpy seeds; each fixture stores a SHA-256 of
its inputs so a test can tell a changed generator from a changed result.

Usage:  python tests/golden/make_golden.py [PREFIX ...]
        (needs the reference checkout; with prefixes, only the fixtures whose
        names start with one of them are rewritten)
"""
import ctypes as C
import hashlib
import os
import random
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("EXCALIBUR_REF", "/root/reference")
REFDIR = os.path.join(ROOT, "oracle", "_ref")


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def p(a):
    return a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------------------
# inputs (shared with the tests through tests/golden/cases.py)
sys.path.insert(0, HERE)
import cases  # noqa: E402


def blas_bound(a, b):
    """The bisection bound exactly as the reference forms it
    (bbtsvd.cpp:936): ||alpha||^2 + ||beta||^2 with the BLAS dnrm2 it links
    (here scipy's OpenBLAS, the library oracle/_ref links)."""
    import glob
    import scipy
    lib = glob.glob(os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs",
                                 "libscipy_openblas-*.so"))[0]
    B = C.CDLL(lib)
    B.scipy_cblas_dnrm2.restype = C.c_double
    B.scipy_cblas_dnrm2.argtypes = [C.c_int, C.c_void_p, C.c_int]
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b if len(b) else np.zeros(1))
    na = B.scipy_cblas_dnrm2(len(a), p(a), 1)
    nb = B.scipy_cblas_dnrm2(len(a) - 1, p(b), 1)
    return na * na + nb * nb


def bidiagonal_fixtures(R):
    out = {}
    for name, (a, b, top_k) in cases.bidiagonal_cases().items():
        k = len(a)
        U = np.zeros(k * top_k)
        V = np.zeros(top_k * k)
        s = np.zeros(k)
        aa, bb = a.copy(), (b.copy() if k > 1 else np.zeros(1))
        R.ref_bidiagonal_svd(C.c_int(k), p(aa), p(bb), p(U), p(V), p(s), C.c_int(top_k))
        mus = cases.sturm_shifts(a, b)
        counts = np.array([R.ref_negative_count(C.c_int(k), p(aa), p(bb), C.c_double(mu)) for mu in mus],
                          dtype=np.int32)
        out[name] = dict(alpha=a, beta=b, top_k=np.int32(top_k), sigma=s[:top_k],
                         bound=np.float64(blas_bound(a, b)),
                         U=U.reshape(k, top_k), V=V.reshape(top_k, k), mus=mus, counts=counts)
    return out


def mask_fixtures(R):
    out = {}
    for name, (x, passes, mask, is_left, seed, fn) in cases.mask_cases().items():
        y = np.ascontiguousarray(x.copy())
        m, n = y.shape
        f = R.ref_givens_mask if fn == "givens" else R.ref_block_shift_mask
        f(C.c_size_t(m), C.c_size_t(n), C.c_size_t(passes), p(y), C.c_int(mask), C.c_int(is_left),
          C.c_uint(seed))
        out[name] = dict(x_sha=sha(x), shape=np.array(x.shape), passes=np.int32(passes),
                         mask=np.int32(mask), is_left=np.int32(is_left), seed=np.uint32(seed),
                         fn=np.array(fn), y=y)
    return out


def run_reference_pipeline(blocks, seed, mode=1, topk=-1, tall=False, y=None):
    """P reference processes over loopback; returns (sigma, FinalU, [FinalVT_c]
    or [w_c] in svd_mode 4, alpha_beta_c0, run_seconds_per_participant).
    ``tall``: the blocks are local_n x m (the reference's layout when
    m > global_n) and FinalU comes back k x m."""
    P = len(blocks)
    m = blocks[0].shape[1] if tall else blocks[0].shape[0]
    ln = [x.shape[0] if tall else x.shape[1] for x in blocks]
    with tempfile.TemporaryDirectory() as td:
        port = random.randint(20000, 40000)
        procs = []
        for c, x in enumerate(blocks):
            np.ascontiguousarray(x, dtype=np.float64).tofile(os.path.join(td, f"Client{c}.mat"))
        if y is not None:
            np.ascontiguousarray(y, dtype=np.float64).tofile(os.path.join(td, "y.mat"))
        env = dict(os.environ, OMP_NUM_THREADS=str(max(1, (os.cpu_count() or 2) // P)))
        for c, x in enumerate(blocks):
            od = os.path.join(td, f"out{c}")
            os.makedirs(od)
            procs.append(subprocess.Popen(
                [os.path.join(REFDIR, "ref_pipeline"), str(c), str(P), str(m), str(ln[c]),
                 str(port), td, td, str(seed), str(mode), str(topk), od],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, env=env, cwd=td))
        for pr in procs:
            if pr.wait(timeout=600) != 0:
                raise RuntimeError("reference participant failed")
        sig = np.fromfile(os.path.join(td, "out0", "sigma.bin"))
        k = len(sig)
        U = (np.fromfile(os.path.join(td, "out0", "U.bin")).reshape((k, m) if tall else (m, k))
             if mode not in (3, 4) else None)
        if mode == 4:
            VT = [np.fromfile(os.path.join(td, f"out{c}", "w.bin")) for c in range(P)]
        else:
            VT = ([np.fromfile(os.path.join(td, f"out{c}", "VT.bin")).reshape(k, ln[c])
                   for c in range(P)] if mode != 2 else None)
        abf = os.path.join(td, "out0", "ab.bin")
        ab = np.fromfile(abf) if os.path.exists(abf) else np.zeros(0)
        secs = [float(open(os.path.join(td, f"out{c}", "time.txt")).read().split()[0]) for c in range(P)]
    return sig, U, VT, ab, secs


def pipeline_fixtures():
    out = {}
    for name, (blocks, seed) in cases.pipeline_cases().items():
        sig, U, VT, ab, secs = run_reference_pipeline(blocks, seed)
        d = dict(x_sha=sha(*blocks), seed=np.uint32(seed), sigma=sig, U=U, ab=ab)
        for c, v in enumerate(VT):
            d[f"VT{c}"] = v
        out[name] = d
    base = cases.pipeline_cases()
    for name, (case, mode, topk) in cases.pipeline_mode_cases().items():
        blocks, seed = base[case]
        sig, U, VT, ab, secs = run_reference_pipeline(blocks, seed, mode=mode, topk=topk)
        d = dict(x_sha=sha(*blocks), seed=np.uint32(seed), sigma=sig, svd_mode=np.int32(mode), top_k=np.int32(topk))
        if U is not None:
            d["U"] = U
        for c, v in enumerate(VT or []):
            d[f"VT{c}"] = v
        out[name] = d
    tall = cases.tall_cases()
    for name, (blocks, seed, y) in tall.items():
        sig, U, VT, ab, secs = run_reference_pipeline(blocks, seed, tall=True)
        d = dict(x_sha=sha(*blocks), seed=np.uint32(seed), sigma=sig, U=U, ab=ab)
        for c, v in enumerate(VT):
            d[f"VT{c}"] = v
        out[name] = d
    for name, (case, mode, topk) in cases.tall_mode_cases().items():
        blocks, seed, y = tall[case]
        sig, U, VT, ab, secs = run_reference_pipeline(blocks, seed, mode=mode, topk=topk, tall=True,
                                                      y=y if mode == 4 else None)
        d = dict(x_sha=sha(*blocks, y), seed=np.uint32(seed), sigma=sig, svd_mode=np.int32(mode),
                 top_k=np.int32(topk))
        if U is not None:
            d["U"] = U
        for c, v in enumerate(VT or []):
            d[f"w{c}" if mode == 4 else f"VT{c}"] = v
        out[name] = d
    for name, (blocks, seed) in cases.square_cases().items():
        for mode in (1, 0):
            sig, U, VT, ab, secs = run_reference_pipeline(blocks, seed, mode=mode)
            d = dict(x_sha=sha(*blocks), seed=np.uint32(seed), sigma=sig, U=U, ab=ab, svd_mode=np.int32(mode))
            for c, v in enumerate(VT):
                d[f"VT{c}"] = v
            out[f"{name}_mode{mode}"] = d
    return out


def step_fixtures(R):
    """The reference's per-step helpers (bbtsvd.cpp:54-164, 970-978) on the
    step cases, each exactly as the reference computes it."""
    out = {}
    for name, (a, b, oi, kt, hx, inc, (cr, sr)) in cases.step_cases().items():
        n = len(a)
        aa, bb = a.copy(), (b.copy() if n > 1 else np.zeros(1))
        l, d = np.zeros(max(n - 1, 1)), np.zeros(n)
        R.ref_ldl(C.c_int(n), p(aa), p(bb), p(l), p(d))
        sig = np.linalg.svd(np.diag(a) + np.diag(b, 1), compute_uv=False)
        omega = float(sig[oi])
        tau = omega * omega
        lp, dp, s = np.zeros(max(n - 1, 1)), np.zeros(n), np.zeros(n)
        R.ref_dstqds(C.c_int(n), p(l), p(d), C.c_double(tau), p(lp), p(dp), p(s))
        up, rp, pp = np.zeros(max(n - 1, 1)), np.zeros(n), np.zeros(n)
        R.ref_dpqds(C.c_int(n), p(l), p(d), C.c_double(tau), p(up), p(rp), p(pp))
        vi = np.zeros(2 * n)
        R.ref_inverse_iteration(C.c_int(n), C.c_int(kt), p(lp), p(up), p(vi), C.c_int(2))
        cnt = 3
        v, u = np.zeros(n), np.zeros(n * cnt)
        R.ref_one_pair(C.c_int(n), C.c_int(cnt), C.c_double(omega), p(l), p(d), p(aa), p(bb), p(v), p(u))
        hxo = hx.copy()
        beta = np.zeros(1)
        R.ref_generate_house(C.c_int(len(hx) // inc), p(hxo), C.c_int(inc), p(beta))
        x2, y2 = a.copy(), np.resize(b, n).copy()
        R.ref_mmap_drot(C.c_size_t(n), p(x2), C.c_size_t(1), p(y2), C.c_size_t(1), C.c_double(cr), C.c_double(sr))
        out[name] = dict(alpha=a, beta=b, omega=np.float64(omega), twist=np.int32(kt), l=l[:n - 1], d=d,
                         lp=lp[:n - 1], dp=dp, s=s, up=up[:n - 1], rp=rp, p=pp, vi=vi, v=v, u=u, house_in=hx,
                         house_inc=np.int32(inc), house_out=hxo, house_beta=beta, drot_c=np.float64(cr),
                         drot_s=np.float64(sr), drot_x=x2, drot_y=y2)
    return out


def generator_fixtures(R):
    """The reference's random orthogonal matrix generators and shuffle_matrix
    (bbtsvd.cpp:301-331, 370-427) on small shapes, each with the next rand()
    value after the call (the glibc state the reference leaves behind)."""
    R.ref_rand.restype = C.c_int
    out = {}
    for name, (layout, m, seed) in {"house_row7": (101, 7, 5), "house_col6": (102, 6, 9)}.items():
        house, tau = np.zeros(m * m), np.zeros(max(m - 1, 1))
        R.ref_random_orthogonal_house(C.c_int(layout), C.c_size_t(m), p(house), p(tau), C.c_uint(seed))
        out[name] = dict(layout=np.int32(layout), m=np.int64(m), seed=np.uint32(seed), house=house, tau=tau,
                         rand_after=np.int64(R.ref_rand()))
    for name, (m, n, seed) in {"orth_tall9x4": (9, 4, 3), "orth_wide4x9": (4, 9, 11)}.items():
        x = np.zeros(m * n)
        R.ref_random_orthogonal(C.c_size_t(m), C.c_size_t(n), p(x), C.c_uint(seed))
        out[name] = dict(m=np.int64(m), n=np.int64(n), seed=np.uint32(seed), x=x, rand_after=np.int64(R.ref_rand()))
    rng = np.random.default_rng(17)
    for name, (m, n, seed, left, unsh) in {"shuffle_left7x5": (7, 5, 21, 1, 0), "unshuffle_left7x5": (7, 5, 21, 1, 1),
                                           "shuffle_right6x9": (6, 9, 8, 0, 0), "unshuffle_right6x9": (6, 9, 8, 0, 1),
                                           "shuffle_left8x3": (8, 3, 2, 1, 0)}.items():
        x0 = rng.standard_normal(m * n)
        x = x0.copy()
        R.ref_shuffle_matrix(C.c_size_t(m), C.c_size_t(n), p(x), C.c_uint(seed), C.c_int(left), C.c_int(unsh))
        out[name] = dict(m=np.int64(m), n=np.int64(n), seed=np.uint32(seed), is_left=np.int32(left),
                         unshuffle=np.int32(unsh), x_in=x0, x_out=x, rand_after=np.int64(R.ref_rand()))
    return out


def other_mask_fixtures(R):
    """The masks of bbtsvd.hpp off the opt_control 1/3 path (bbtsvd.cpp:190-299,
    429-531, 670-726) on small blocks, each with the next rand() value after
    the call."""
    R.ref_rand.restype = C.c_int
    out = {}
    rng = np.random.default_rng(29)
    for name, (fn, m, n, size, rounds, mask, left, seed) in cases.OTHER_MASK_CASES.items():
        x0 = rng.standard_normal(m * n)
        x = x0.copy()
        args = (C.c_size_t(m), C.c_size_t(n), C.c_size_t(size))
        tail = (p(x), C.c_int(mask), C.c_int(left), C.c_uint(seed))
        if fn == "naive":
            R.ref_naive_givens(*args, *tail)
        elif fn == "cached":
            R.ref_givens_cached(*args, *tail)
        elif fn == "block":
            R.ref_block_mask(*args, *tail)
        elif fn == "shufblock":
            R.ref_shuffle_block_mask(*args, C.c_int(rounds), *tail)
        elif fn == "house":
            R.ref_house_mask(*args, *tail)
        else:
            R.ref_householder_reflector_mask(*args, *tail)
        out[name] = dict(x_in=x0, x_out=x, rand_after=np.int64(R.ref_rand()))
    return out


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={REF}"], check=True)
    R = C.CDLL(os.path.join(REFDIR, "libref_capi.so"))
    R.ref_negative_count.restype = C.c_int
    R.ref_set_threads(1)
    fx = {}
    groups = (("bidiag", bidiagonal_fixtures), ("mask", mask_fixtures), ("step", step_fixtures),
              ("gen", generator_fixtures), ("omask", other_mask_fixtures), ("pipe", lambda R: pipeline_fixtures()))
    keep = sys.argv[1:]
    for grp, fn in groups:
        if keep and not any(k.startswith(grp) for k in keep):
            continue
        d = fn(R)
        for name, arrs in d.items():
            fx[f"{grp}__{name}"] = arrs
    fx = {k: v for k, v in fx.items() if not keep or any(k.startswith(p) for p in keep)}
    for key, arrs in fx.items():
        np.savez_compressed(os.path.join(HERE, f"{key}.npz"), **arrs)
    print(f"wrote {len(fx)} fixtures to {HERE}")


if __name__ == "__main__":
    main()
