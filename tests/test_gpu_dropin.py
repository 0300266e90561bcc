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
import time

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
            # output to files, never to pipes nobody drains while the peers wait on each other
            with open(os.path.join(od, "stderr.txt"), "wb") as ef:
                procs.append(subprocess.Popen([EXE, str(c), str(P), str(m), str(ln[c]), str(port), td, td,
                                               str(seed), str(mode), str(topk), od, str(opt)],
                                              stdout=subprocess.DEVNULL, stderr=ef, env=env, cwd=td))
        # a participant that fails leaves its peers waiting on their sockets:
        # end them all as soon as one fails, and bound the whole case
        deadline = time.monotonic() + 120
        while any(pr.poll() is None for pr in procs):
            if any(pr.returncode not in (None, 0) for pr in procs) or time.monotonic() > deadline:
                for pr in procs:
                    if pr.poll() is None:
                        pr.kill()
                break
            time.sleep(0.05)
        errs = []
        for c, pr in enumerate(procs):
            pr.wait()
            if pr.returncode != 0:
                e = open(os.path.join(td, f"out{c}", "stderr.txt"), "rb").read()
                errs.append(f"participant {c} rc={pr.returncode}: " + e.decode(errors="replace")[-500:])
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


def _exclusive_process():
    """True when the GPU admits one process at a time (compute mode
    EXCLUSIVE_PROCESS): P participants as P processes cannot all hold a
    context, so only single-participant runs are possible there."""
    try:
        out = subprocess.run(["nvidia-smi", "-i", os.environ.get("BBT_DEVICE", "0"), "--query-gpu=compute_mode",
                              "--format=csv,noheader"], capture_output=True, text=True, timeout=20).stdout
        return "exclusive" in out.lower()
    except Exception:
        return False


@pytest.fixture(scope="module")
def exe():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    assert os.path.exists(EXE), "oracle/_ref/ref_pipeline_b200 missing: make -C oracle dropin REF=<Excalibur checkout>"
    return EXE


@pytest.fixture(scope="module")
def multi(exe):
    """Several participant processes on this GPU."""
    if _exclusive_process():
        pytest.skip("the GPU is in EXCLUSIVE_PROCESS compute mode: one process per GPU, so the multi-participant "
                    "drop-in runs cannot share it (the single-participant runs below cover the boundary)")
    return exe


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
def test_reference_client_on_library(multi, golden, name):
    blocks, seed = cases.pipeline_cases()[name]
    sig, U, VT = run_dropin(blocks, seed)
    _compare(golden(f"pipe__{name}"), sig, U, VT, 1)


@pytest.mark.parametrize("name", sorted(cases.pipeline_mode_cases()))
def test_reference_client_on_library_modes(multi, golden, name):
    case, mode, topk = cases.pipeline_mode_cases()[name]
    blocks, seed = cases.pipeline_cases()[case]
    sig, U, VT = run_dropin(blocks, seed, mode=mode, topk=topk)
    _compare(golden(f"pipe__{name}"), sig, U, VT, mode)


@pytest.mark.parametrize("name", sorted(cases.tall_cases()) + sorted(cases.tall_mode_cases()))
def test_reference_client_on_library_tall(exe, golden, name):
    tall, modes = cases.tall_cases(), cases.tall_mode_cases()
    case, mode, topk = (name, 1, -1) if name in tall else modes[name]
    blocks, seed, y = tall[case]
    if len(blocks) > 1 and _exclusive_process():
        pytest.skip("EXCLUSIVE_PROCESS GPU: one participant process at a time")
    sig, U, VT = run_dropin(blocks, seed, mode=mode, topk=topk, tall=True, y=y if mode == 4 else None)
    _compare(golden(f"pipe__{name}"), sig, U, VT, mode)


@pytest.mark.parametrize("name", sorted(cases.square_cases()))
@pytest.mark.parametrize("mode", [1, 0])
def test_reference_client_on_library_square(exe, golden, mode, name):
    blocks, seed = cases.square_cases()[name]
    if len(blocks) > 1 and _exclusive_process():
        pytest.skip("EXCLUSIVE_PROCESS GPU: one participant process at a time")
    sig, U, VT = run_dropin(blocks, seed, mode=mode)
    _compare(golden(f"pipe__{name}_mode{mode}"), sig, U, VT, mode)
