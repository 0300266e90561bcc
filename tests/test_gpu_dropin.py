"""The drop-in boundary exercised for real: the reference's own
DecentralizedClient (Excalibur src/client.cpp, src/utils.cpp, the logger)
compiled WITHOUT its src/bbtsvd.cpp and linked against libexcalibur_b200.so,
which supplies every bbtsvd.hpp function it calls (block_shift_mask,
negative_count, bisection_singular_values,
bidiagonal_bisection_twisted_svd) with the same C++ signatures
(oracle/Makefile, target dropin).  P participants run as P processes over
loopback TCP, exactly as the reference runs; its run() is unmodified.  The
outputs must equal the reference's own outputs (golden fixtures written by
the reference's build with its own bbtsvd.cpp): the masks and the bisection
are bit-exact, so every bidiagonal, and hence every singular value, is the
reference's bit for bit; the twisted vectors agree to rounding."""
import os
import random
import subprocess
import tempfile

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "ref_pipeline_b200")


def run_dropin(blocks, seed, mode=1, topk=-1, tall=False, y=None, opt=3):
    P = len(blocks)
    m = blocks[0].shape[1] if tall else blocks[0].shape[0]
    ln = [x.shape[0] if tall else x.shape[1] for x in blocks]
    with tempfile.TemporaryDirectory() as td:
        for c, x in enumerate(blocks):
            np.ascontiguousarray(x, dtype=np.float64).tofile(os.path.join(td, f"Client{c}.mat"))
        if y is not None:
            np.ascontiguousarray(y, dtype=np.float64).tofile(os.path.join(td, "y.mat"))
        env = dict(os.environ, OMP_NUM_THREADS="2", OPENBLAS_NUM_THREADS="2")
        port = random.randint(20000, 40000)
        procs = []
        for c in range(P):
            od = os.path.join(td, f"out{c}")
            os.makedirs(od)
            procs.append(subprocess.Popen([EXE, str(c), str(P), str(m), str(ln[c]), str(port), td, td, str(seed),
                                           str(mode), str(topk), od, str(opt)],
                                          stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, env=env, cwd=td))
        errs = []
        for pr in procs:
            try:
                _, e = pr.communicate(timeout=300)
            except subprocess.TimeoutExpired:
                pr.kill()
                _, e = pr.communicate()
            if pr.returncode != 0:
                errs.append(e.decode(errors="replace")[-500:])
        assert not errs, errs
        sig = np.fromfile(os.path.join(td, "out0", "sigma.bin"))
        k = len(sig)
        U = (np.fromfile(os.path.join(td, "out0", "U.bin")).reshape((k, m) if tall else (m, k))
             if mode not in (3, 4) else None)
        if mode == 4:
            VT = [np.fromfile(os.path.join(td, f"out{c}", "w.bin")) for c in range(P)]
        elif mode == 2:
            VT = None
        else:
            VT = [np.fromfile(os.path.join(td, f"out{c}", "VT.bin")).reshape(k, ln[c]) for c in range(P)]
    return sig, U, VT


@pytest.fixture(scope="module")
def exe():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    assert os.path.exists(EXE), "oracle/_ref/ref_pipeline_b200 missing: make -C oracle dropin REF=<Excalibur checkout>"
    return EXE


def _compare(g, sig, U, VT, mode, key="VT"):
    assert len(sig) == len(g["sigma"])
    assert np.array_equal(sig, g["sigma"]), np.max(np.abs(sig - g["sigma"]) / g["sigma"])
    if mode not in (3, 4):
        assert np.max(np.abs(U - g["U"])) < 1e-12
    if mode == 4:
        for c, w in enumerate(VT):
            assert np.max(np.abs(w - g[f"w{c}"])) < 1e-12 * max(1.0, np.abs(g[f"w{c}"]).max())
    elif mode != 2:
        for c, v in enumerate(VT):
            assert np.max(np.abs(v - g[f"{key}{c}"])) < 1e-12


@pytest.mark.parametrize("name", sorted(cases.pipeline_cases()))
def test_reference_client_on_library(exe, golden, name):
    blocks, seed = cases.pipeline_cases()[name]
    sig, U, VT = run_dropin(blocks, seed)
    _compare(golden(f"pipe__{name}"), sig, U, VT, 1)


@pytest.mark.parametrize("name", sorted(cases.pipeline_mode_cases()))
def test_reference_client_on_library_modes(exe, golden, name):
    case, mode, topk = cases.pipeline_mode_cases()[name]
    blocks, seed = cases.pipeline_cases()[case]
    sig, U, VT = run_dropin(blocks, seed, mode=mode, topk=topk)
    _compare(golden(f"pipe__{name}"), sig, U, VT, mode)


@pytest.mark.parametrize("name", sorted(cases.tall_cases()) + sorted(cases.tall_mode_cases()))
def test_reference_client_on_library_tall(exe, golden, name):
    tall, modes = cases.tall_cases(), cases.tall_mode_cases()
    case, mode, topk = (name, 1, -1) if name in tall else modes[name]
    blocks, seed, y = tall[case]
    sig, U, VT = run_dropin(blocks, seed, mode=mode, topk=topk, tall=True, y=y if mode == 4 else None)
    _compare(golden(f"pipe__{name}"), sig, U, VT, mode)


@pytest.mark.parametrize("mode", [1, 0])
def test_reference_client_on_library_square(exe, golden, mode):
    blocks, seed = cases.square_cases()["sq80"]
    sig, U, VT = run_dropin(blocks, seed, mode=mode)
    _compare(golden(f"pipe__sq80_mode{mode}"), sig, U, VT, mode)
