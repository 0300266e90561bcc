"""Benchmark: decentralized SVD wall time on one B200 (per replica).

Headline workload (c2): 2 participants, each holding a 500,000 x 1,000 FP64
block of X = U diag(s) V^T (U 10^6 x 1000 and V 1000 x 1000 Haar-random,
seeded; s geometric from 1 to 1e-6) -- the reference's short-and-wide branch
with m = 1000 and local_n = 500,000.  One step is the whole pipeline (local
QR, masks, global QR, Ralha bidiagonalisation, bisection + twisted vectors,
back-transforms) on inputs resident in HBM; the 8 GB inputs are larger than
L2, and are restored from a pristine device copy before every step (outside
the timed events).

The three precision modes are timed: plain FP64 (mode 0, the reference's
Householder local QR), mixed (mode 1: BF16x3 tensor-core sketch + FP64
Cholesky-QR refinement) and exact Gram (mode 2: the sketch as a
preconditioner of the exact Gram matrix, computed on the int8 tensor cores by
the Chinese remainder theorem, and products with the implicit Q made exact the
same way); the JSON value is mode 2, the other two sit beside it under
"plain" and "mixed".

The other workloads run after the headline, each under its own key with its
own (smaller) step counts:
  c1  2 participants x 1,000 x 100 N(0,1) (the reference's CPU-runnable case);
  c3  64 participants, rows uniform in [10,000, 200,000] x 512, entries
      N(0,1) x 10^U[-2,2] per participant (the batched local QR);
  c4  one 8,192 x 8,192 matrix with 512 clusters of 16 singular values at
      relative spacing 1e-10, centres log-uniform in [1e-8, 1] (dense SVD);
  c5  4 participants x 2,000 x 1,000,000 (64 GB): rank 50 with singular
      values 1e3 .. 10 plus N(0, 1e-3) noise; full spectrum and top-50.
Every result carries its error against an FP64 oracle of the stored inputs.

Prints one JSON line (rank 0).  --impl reference times the reference's own
CPU implementation (oracle/_ref, built from the reference's sources) on the
same c2 workload at full size.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # name: (participants, m, local_n (first participant; see make_blocks), spectrum)
    "c2": (2, 1000, 500_000, "geometric"),
    "c1": (2, 100, 1000, "gaussian"),
    "c3": (64, 512, 0, "scaled"),   # rows per participant uniform in [10,000, 200,000]
    "c5": (4, 2000, 1_000_000, "lowrank"),
}
C4_N = 8192
EXTRAS = ("c1", "c3", "c4", "c5")


def c3_rows(seed=0):
    """Row counts of the 64 participants of c3 (seeded)."""
    return [int(r) for r in np.random.default_rng(seed).integers(10_000, 200_001, 64)]


METRIC = "SVD wall-s at rel err <=1e-10 vs FP64 oracle"
PRECISION = {"plain": 0, "mixed": 1, "exact": 2}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    p.add_argument("--rows", type=int, default=0, help="override local_n (smaller runs)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--extras", default="all",
                   help="comma list of the other workloads timed after the headline (c1,c3,c4,c5), "
                        "'all' or 'none'")
    p.add_argument("--only", default=None, choices=list(EXTRAS),
                   help="run just this one of the other workloads (no headline line): for profiling")
    p.add_argument("--c4-n", type=int, default=C4_N, help="order of the c4 dense matrix (smaller runs)")
    p.add_argument("--no-check", action="store_true",
                   help="skip the FP64 oracle and the accuracy check (launch-list captures of the pipeline alone)")
    p.add_argument("--precision", default="all", choices=["both", "mixed", "plain", "exact", "all"],
                   help="all: plain FP64, mixed (mode 1) and exact Gram (mode 2), the JSON value is the last; "
                        "both: plain then mixed")
    return p.parse_args()


# ---------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, gpu):
        self.gpu, self.samples, self.stop = gpu, [], threading.Event()

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.t.join(timeout=10)

    def summary(self):
        sm = [float(s[0]) for s in self.samples if s and s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if len(s) > 1 and s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 3 + i and s[3 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ---------------------------------------------------------------- data
def make_blocks(torch, dev, P, m, n, spectrum, seed=0):
    """Participant blocks X_c (m x n row-major), X = [X_0 | X_1 | ...]."""
    g = torch.Generator(device=dev).manual_seed(seed)
    if spectrum == "gaussian":
        return [torch.randn(m, n, generator=g, device=dev, dtype=torch.float64) for _ in range(P)], None
    if spectrum == "scaled":   # c3: N(0,1) entries times 10^U[-2,2] per participant
        rows = c3_rows(seed)
        scl = np.random.default_rng(seed + 1).uniform(-2.0, 2.0, P)
        return [torch.randn(m, r, generator=g, device=dev, dtype=torch.float64) * float(10.0 ** f)
                for r, f in zip(rows, scl)], None
    G = torch.randn(P * n, m, generator=g, device=dev, dtype=torch.float64)
    Q, R = torch.linalg.qr(G)
    Q *= torch.sign(torch.diagonal(R))
    del G, R
    H = torch.randn(m, m, generator=g, device=dev, dtype=torch.float64)
    V, R = torch.linalg.qr(H)
    V *= torch.sign(torch.diagonal(R))
    s = torch.logspace(0, -6, m, dtype=torch.float64, device=dev)
    # row-stacked X_s = Q diag(s) V^T; participant c holds (rows of c)^T = V diag(s) Q_c^T
    blocks = [(V * s) @ Q[c * n:(c + 1) * n].T for c in range(P)]
    del Q
    return [b.contiguous() for b in blocks], s


class LowRank:
    """c5's participants: X = A diag(s) B^T + N(0, sigma_noise^2), A (m x rank)
    and B (P n x rank) orthonormal (seeded Haar), s geometric from s_hi to
    s_lo; block c holds columns c n .. (c+1) n.  fill(c, out) rewrites block c
    identically every time (its noise comes from its own seeded generator)."""

    def __init__(self, torch, dev, P, m, n, rank=50, s_hi=1e3, s_lo=10.0, noise=1e-3, seed=0):
        self.torch, self.dev, self.P, self.m, self.n, self.noise, self.seed = torch, dev, P, m, n, noise, seed
        g = torch.Generator(device=dev).manual_seed(seed)
        A, R = torch.linalg.qr(torch.randn(m, rank, generator=g, device=dev, dtype=torch.float64))
        A *= torch.sign(torch.diagonal(R))
        B, R = torch.linalg.qr(torch.randn(P * n, rank, generator=g, device=dev, dtype=torch.float64))
        B *= torch.sign(torch.diagonal(R))
        self.s = torch.logspace(math.log10(s_hi), math.log10(s_lo), rank, dtype=torch.float64, device=dev)
        self.As = A * self.s
        self.B = B

    def fill(self, c, out):
        torch = self.torch
        g = torch.Generator(device=self.dev).manual_seed(self.seed + 1000 + c)
        torch.randn(out.shape, generator=g, dtype=torch.float64, device=self.dev, out=out)
        out.mul_(self.noise)
        out.addmm_(self.As, self.B[c * self.n:(c + 1) * self.n].T)


def fp64_oracle(torch, blocks):
    """FP64 SVD of the stored X on the GPU (cuSOLVER Householder QR of every
    block, QR of the stacked R factors, SVD): the measurement's accuracy
    oracle, not part of the timed path.  X^T = Q R, so X = R^T Q^T."""
    Rs = []
    for b in blocks:
        Rs.append(torch.linalg.qr(b.T, mode="r")[1])
        torch.cuda.empty_cache()
    R = torch.linalg.qr(torch.cat(Rs, dim=0), mode="r")[1]
    Ur, s, Vh = torch.linalg.svd(R.T)
    return s, Ur


def well_posed(torch, s_ref, k):
    gap = torch.full_like(s_ref[:k], float("inf"))
    d = s_ref[:k - 1] - s_ref[1:k]
    gap[1:] = torch.minimum(gap[1:], d)
    gap[:-1] = torch.minimum(gap[:-1], d)
    if k < len(s_ref):
        gap[k - 1] = torch.minimum(gap[k - 1], s_ref[k - 1] - s_ref[k])
    return (2.2e-16 * s_ref[0] / gap) <= 1e-10


def accuracy(torch, s_ref, U_ref, s, U, blocks=None, VT=None):
    """sigma relative errors and gap-aware per-vector angles (sine form:
    sin(angle) = || u - (u_ref . u) u_ref ||; arccos of the cosine bottoms out
    near 1.5e-8 in FP64) of the left vectors and, with the blocks and FinalVT,
    of the right vectors against v_ref = X^T u_ref / sigma_ref (normalised)."""
    k = min(len(s), len(s_ref))
    rel = (s[:k] - s_ref[:k]).abs() / s_ref[:k]
    d = (U_ref[:, :k] * U[:, :k]).sum(dim=0)
    ang = torch.linalg.vector_norm(U[:, :k] - U_ref[:, :k] * d, dim=0).clamp(max=1.0).arcsin()
    well = well_posed(torch, s_ref, k)
    out = {"sigma_rel_err_max": float(rel.max()), "sigma_count": int(len(s)),
           "u_angle_max_well_posed": float(ang[well].max()) if bool(well.any()) else None,
           "u_angle_max_all": float(ang.max())}
    if blocks is not None and VT is not None:
        # two passes over the participants: the dot products and norms first,
        # then the residuals v - d v_ref (v_ref recomputed, never held whole)
        dot = torch.zeros(k, dtype=torch.float64, device=s.device)
        nrm = torch.zeros_like(dot)
        for b, v in zip(blocks, VT):
            vr = U_ref[:, :k].T @ b
            dot += (vr * v[:k]).sum(dim=1)
            nrm += (vr * vr).sum(dim=1)
            del vr
        nrm = nrm.sqrt()
        dot /= nrm
        res = torch.zeros_like(dot)
        for b, v in zip(blocks, VT):
            vr = (U_ref[:, :k].T @ b) / nrm[:, None]
            res += ((v[:k] - vr * dot[:, None]) ** 2).sum(dim=1)
            del vr
        vang = res.sqrt().clamp(max=1.0).arcsin()
        out["v_angle_max_well_posed"] = float(vang[well].max()) if bool(well.any()) else None
        out["v_angle_max_all"] = float(vang.max())
    return out


# ---------------------------------------------------------------- reference arm
def write_client_files(torch, blocks, td):
    """The reference's input files: Client<c>.mat, raw float64 row-major
    m x local_n[c] (utils.cpp:237-252)."""
    for c, b in enumerate(blocks):
        b.cpu().numpy().tofile(os.path.join(td, f"Client{c}.mat"))


def reference_run(P, m, ns, td, threads=None, mode=1, top_k=-1):
    """One run of the reference's own pipeline (oracle/_ref/ref_pipeline, P
    processes over loopback TCP) on the Client<c>.mat files in td.  Returns
    (max over participants of the reference's own run() timer, per-phase
    seconds of participant 0, threads used)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_pipeline")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    cores = os.cpu_count() or 1
    threads = threads or max(1, cores // P)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS=str(threads))
    port = 20000 + (os.getpid() * 7 + int(time.time() * 13)) % 20000
    procs = []
    with tempfile.TemporaryDirectory(dir=td) as od:
        for c in range(P):
            oc = os.path.join(od, f"o{c}")
            os.makedirs(oc)
            procs.append(subprocess.Popen([exe, str(c), str(P), str(m), str(ns[c]), str(port), td, od, "0",
                                           str(mode), str(top_k), oc],
                                          stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, env=env, cwd=od))
        for pr in procs:
            if pr.wait(timeout=1800) != 0:
                raise RuntimeError("reference participant failed")
        times = [list(map(float, open(os.path.join(od, f"o{c}", "time.txt")).read().split())) for c in range(P)]
    total = max(t[0] for t in times)
    phases = dict(zip(("total", "local_qr", "global_qr", "apply_mask", "exchange", "bi_diag", "bsvd", "combine",
                       "comm"), times[0]))
    return total, phases, min(threads * P, cores)


def reference_data(args):
    """The headline workload's blocks (the GPU arm's generator, on the GPU when
    there is one) written as the reference's input files.  Returns (tempdir
    object, P, m, local_n list)."""
    import torch
    P, m, n, spectrum = CONFIGS[args.config]
    if args.rows:
        n = args.rows
    dev = torch.device("cuda", 0) if torch.cuda.is_available() else torch.device("cpu")
    blocks, _ = make_blocks(torch, dev, P, m, n, spectrum, seed=0)
    td = tempfile.TemporaryDirectory(dir=os.environ.get("EXCALIBUR_BENCH_TMP"))
    write_client_files(torch, blocks, td.name)
    ns = [int(b.shape[1]) for b in blocks]
    del blocks
    if dev.type == "cuda":
        torch.cuda.empty_cache()
    return td, P, m, ns


# ---------------------------------------------------------------- our arm
def cublas_dgemm_peak(torch, dev):
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2 * 8192 ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best


def cublas_int8_peak(torch, dev):
    """Dense int8 tensor-core throughput of a library GEMM (torch._int_mm,
    8192^3, int8 x int8 -> int32), best of 5: the denominator of the CRT
    kernel's roofline.  None where the library has no int8 path."""
    try:
        a = torch.randint(-100, 100, (8192, 8192), dtype=torch.int8, device=dev)
        b = torch.randint(-100, 100, (8192, 8192), dtype=torch.int8, device=dev).T.contiguous().T
        for _ in range(2):
            torch._int_mm(a, b)
        torch.cuda.synchronize()
        best = 0.0
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = max(best, 2 * 8192 ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
        return best
    except Exception:
        return None


def max_over_ranks(torch, value, device, world):
    """The largest of every rank's value (a collective every rank calls in
    the same order): the job-level time of replicas timed independently."""
    if world <= 1:
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t)


def time_fedsvd(torch, ctx, blocks, restore, pub, priv, prec, warmup, steps, dev, world, top_k=-1,
                check=None):
    """warmup + steps runs of the pipeline; the device time of a step is the
    sum of its stage events (CUDA events on the library's stream).  restore()
    rewrites the inputs before every run (outside the events); check(out) is
    the accuracy of the last warm-up run."""
    acc = None
    for i in range(warmup):
        restore()
        torch.cuda.synchronize()
        out = ctx.fedsvd(blocks, pub, priv, precision=prec, top_k=top_k)
        if check is not None and i == warmup - 1:
            acc = check(out)
        del out
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    l0 = ctx.launches()
    times, stage = [], {}
    ctx.profile(True)
    with Clocks(dev.index) as clk:
        for _ in range(steps):
            restore()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = ctx.fedsvd(blocks, pub, priv, precision=prec, top_k=top_k)      # synchronises before returning
            times.append(time.perf_counter() - t0)
            for kk, v in ctx.stage_ms().items():
                stage[kk] = stage.get(kk, 0.0) + v / steps
            del out
    prof = ctx.profile_get()
    ctx.profile(False)
    launches = (ctx.launches() - l0) // steps
    torch.cuda.synchronize()
    sec = max_over_ranks(torch, sum(stage.values()) / 1e3, dev, world)
    return {"sec": sec, "host_sec": statistics.median(times), "stage_ms": stage, "acc": acc,
            "launches": launches, "prof": prof, "clocks": clk.summary()}


def run_ours(args, rank, world):
    """Times the headline pipeline at each requested precision (plain FP64
    first, then mixed, then exact Gram); returns {precision: result} plus the
    end-to-end measurement of the headline precision."""
    import torch
    import excalibur_b200 as eb
    P, m, n, spectrum = CONFIGS[args.config]
    if args.rows:
        n = args.rows
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    ctx = eb.Context(dev.index)
    blocks, s_gen = make_blocks(torch, dev, P, m, n, spectrum, seed=0)
    pristine = [b.clone() for b in blocks]
    s_ref, U_ref = (None, None) if args.no_check else fp64_oracle(torch, pristine)
    pub, priv = eb.reference_seeds(0, P)
    batched = sum(1 for b in pristine if b.shape[1] // m > 5) >= 8
    precisions = {"both": ["plain", "mixed"], "plain": ["plain"], "mixed": ["mixed"], "exact": ["exact"],
                  "all": ["plain", "mixed", "exact"]}[args.precision]

    def restore():
        for b, p0 in zip(blocks, pristine):
            b.copy_(p0)

    def check(out):
        return accuracy(torch, s_ref, U_ref, out[0], out[1], pristine, out[2])

    out_all = {}
    for pname in precisions:
        prec = PRECISION[pname]
        tuned = ctx.fedsvd_tune(m, [b.shape[1] for b in pristine], precision=prec) if batched else None
        r = time_fedsvd(torch, ctx, blocks, restore, pub, priv, prec, args.warmup, args.steps, dev, world,
                        check=None if args.no_check else check)
        r["tuned"] = tuned
        out_all[pname] = r
    res = {"runs": out_all, "head": precisions[-1]}
    if rank == 0:
        res["dgemm_peak"] = cublas_dgemm_peak(torch, dev)
        res["int8_peak"] = cublas_int8_peak(torch, dev)
    if not args.no_e2e:
        # end to end through the host-pointer C-ABI entry: pinned host inputs,
        # H2D + pipeline + D2H inside the timed call
        prec = PRECISION[res["head"]]
        hb = [p0.cpu().pin_memory().numpy() for p0 in pristine]
        del blocks
        torch.cuda.empty_cache()
        outbuf = (torch.empty(m, dtype=torch.float64).pin_memory().numpy(),
                  torch.empty(m * m, dtype=torch.float64).pin_memory().numpy(),
                  [torch.empty(m * p0.shape[1], dtype=torch.float64).pin_memory().numpy() for p0 in pristine])
        ctx.fedsvd_host(hb, pub, priv, precision=prec, out=outbuf)     # warm
        et = []
        for _ in range(max(1, min(args.steps, 3))):
            t0 = time.perf_counter()
            sg, Ug, VTg = ctx.fedsvd_host(hb, pub, priv, precision=prec, out=outbuf)
            et.append(time.perf_counter() - t0)
        k = len(sg)
        res["e2e"] = {"value": max_over_ranks(torch, statistics.median(et), dev, world), "unit": "s",
                      "precision": res["head"],
                      "h2d_bytes_per_step": int(sum(h.nbytes for h in hb)),
                      "d2h_bytes_per_step": int(8 * (k + m * k + k * sum(h.shape[1] for h in hb)))}
        del hb, outbuf
    del pristine
    ctx.close()
    torch.cuda.empty_cache()
    return res


def summarize(o, dgemm_peak, int8_peak, head=False):
    d = {"value": o["sec"], "unit": "s", "accuracy": o["acc"], "stage_ms": o["stage_ms"],
         "gpu_launches": o["launches"], "roofline": roofline(o["prof"], dgemm_peak, int8_peak),
         "kernel_classes": {k: {"ms": v[0], "launches": v[1]} for k, v in o["prof"].items() if v[1]}}
    if not head:
        d["clocks"] = o["clocks"]
    return d


# ---------------------------------------------------------------- other workloads
def extra_blocks(args, rank, world, name, modes, warmup, steps, dgemm_peak, int8_peak):
    """c1 / c3: the pipeline in the given precision modes, with its oracle."""
    import torch
    import excalibur_b200 as eb
    P, m, n, spectrum = CONFIGS[name]
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    ctx = eb.Context(dev.index)
    blocks, _ = make_blocks(torch, dev, P, m, n, spectrum, seed=0)
    pristine = [b.clone() for b in blocks]
    s_ref, U_ref = fp64_oracle(torch, pristine)
    pub, priv = eb.reference_seeds(0, P)
    batched = sum(1 for b in pristine if b.shape[1] // m > 5) >= 8

    def restore():
        for b, p0 in zip(blocks, pristine):
            b.copy_(p0)

    out = {"workload": workload_name(name), "warmup": warmup, "steps": steps}
    for pname in modes:
        prec = PRECISION[pname]
        tuned = ctx.fedsvd_tune(m, [b.shape[1] for b in pristine], precision=prec) if batched else None
        r = time_fedsvd(torch, ctx, blocks, restore, pub, priv, prec, warmup, steps, dev, world,
                        check=lambda o: accuracy(torch, s_ref, U_ref, o[0], o[1], pristine, o[2]))
        out[pname] = summarize(r, dgemm_peak, int8_peak)
        if tuned is not None:
            out[pname]["batched_local_qr"] = {"streams": tuned[0], "panel_width": tuned[1], "tuning_ms": tuned[2]}
    if "plain" in out and "exact" in out:
        out["speedup_exact_vs_plain"] = out["plain"]["value"] / out["exact"]["value"]
    del blocks, pristine
    ctx.close()
    torch.cuda.empty_cache()
    return out


def clustered_spectrum(rng, clusters, size, gap=1e-10, lo=1e-8, hi=1.0):
    c = np.exp(rng.uniform(np.log(lo), np.log(hi), clusters))
    return np.sort(np.concatenate([ci * (1.0 + gap * np.arange(size)) for ci in c]))[::-1]


def extra_c4(rank, world, warmup, steps, n=C4_N):
    """c4: the dense SVD of one 8192^2 matrix X = Ux diag(s) Vx^T (Haar Ux, Vx)
    with 512 clusters of 16 values at relative spacing 1e-10.  Oracle: the
    singular values of the stored X by cuSOLVER (FP64); cluster subspaces
    against Ux / Vx at the gap-aware bar max(1e-8, 100 eps ||X|| / gap)."""
    import torch
    import excalibur_b200 as eb
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    ctx = eb.Context(dev.index)
    rng = np.random.default_rng(4)
    s = clustered_spectrum(rng, n // 16, 16)
    sv = torch.as_tensor(s.copy(), device=dev)
    g = torch.Generator(device=dev).manual_seed(4)

    def haar():
        q, r = torch.linalg.qr(torch.randn(n, n, generator=g, device=dev, dtype=torch.float64))
        return q * torch.sign(torch.diagonal(r))

    Ux, Vx = haar(), haar()
    X0 = (Ux * sv) @ Vx.T
    t0 = time.perf_counter()
    so = torch.linalg.svdvals(X0)
    torch.cuda.synchronize()
    oracle_s = time.perf_counter() - t0
    X = torch.empty_like(X0)
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream)
    res = None
    for _ in range(warmup):
        X.copy_(X0)
        res = ctx.svd_dense(X)
    sg, U, VT = res
    rel = (sg - so).abs() / so
    big = so > 1e-5 * so[0]
    # cluster subspaces (sine form) against the generating Ux, Vx: a cluster is
    # well posed when eps ||X|| / gap <= 1e-10 (gap to the neighbouring
    # clusters), the criterion of the per-vector checks elsewhere; every
    # cluster is also measured against the backward-error bar eps n ||X|| / gap
    eps = 2.2e-16
    well_u = well_v = 0.0
    worst_u = worst_v = 0.0
    nwell = 0
    for c in range(n // 16):
        grp = slice(16 * c, 16 * c + 16)
        lo = s[16 * c + 15] - (s[16 * c + 16] if 16 * c + 16 < n else 0.0)
        hi = (s[16 * c - 1] - s[16 * c]) if c > 0 else np.inf
        gap = min(lo, hi)
        A, B = U[:, grp], Ux[:, grp]
        su = torch.linalg.matrix_norm(A - B @ (B.T @ A), ord=2).item()
        A, B = VT[grp].T, Vx[:, grp]
        sv_ = torch.linalg.matrix_norm(A - B @ (B.T @ A), ord=2).item()
        bar = max(1e-8, eps * n * s[0] / gap)
        worst_u, worst_v = max(worst_u, su / bar), max(worst_v, sv_ / bar)
        if eps * s[0] / gap <= 1e-10:
            nwell += 1
            well_u, well_v = max(well_u, su), max(well_v, sv_)
    orth = float((U.T @ U - torch.eye(n, dtype=torch.float64, device=dev)).abs().max())
    acc = {"sigma_rel_err_max_above_1e-5": float(rel[big].max()),
           "sigma_abs_err_max_over_smax": float(((sg - so).abs() / so[0]).max()),
           "cluster_u_angle_max_well_posed": well_u, "cluster_v_angle_max_well_posed": well_v,
           "well_posed_clusters": nwell, "clusters": n // 16,
           "cluster_u_angle_worst_over_backward_bar": worst_u, "cluster_v_angle_worst_over_backward_bar": worst_v,
           "u_orthogonality_max": orth, "sigma_count": int(len(sg)), "oracle": "cuSOLVER FP64 svdvals of the "
           "stored X (%.1f s); FP64 storage bounds relative accuracy below ~1e-5 sigma_max; cluster subspaces "
           "against the generating Ux, Vx" % oracle_s}
    del res, sg, U, VT
    torch.cuda.synchronize()
    times = []
    ctx.profile(True)
    with Clocks(dev.index) as clk:
        for _ in range(steps):
            X.copy_(X0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = ctx.svd_dense(X)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
            del out
    prof = ctx.profile_get()
    ctx.profile(False)
    ctx.set_stream(None)
    ctx.close()
    del X, X0, Ux, Vx
    torch.cuda.empty_cache()
    return {"workload": workload_name("c4", n), "warmup": warmup, "steps": steps,
            "value": max_over_ranks(torch, statistics.median(times), dev, world), "unit": "s",
            "accuracy": acc, "clocks": clk.summary(),
            "kernel_classes": {k: {"ms": v[0] / steps, "launches": v[1] // steps} for k, v in prof.items() if v[1]}}


def extra_c5(rank, world, warmup, steps, dgemm_peak, int8_peak, modes=("exact", "mixed", "plain")):
    """c5: 4 participants x 2000 x 10^6 (64 GB), rank 50 plus noise; the full
    spectrum in each precision mode and the top 50 in the exact-Gram mode.
    Inputs are regenerated on the device before every run (plain and mixed
    overwrite them; outside the timed events)."""
    import torch
    import excalibur_b200 as eb
    P, m, n, _ = CONFIGS["c5"]
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    gen = LowRank(torch, dev, P, m, n)
    blocks = [torch.empty(m, n, dtype=torch.float64, device=dev) for _ in range(P)]
    for c, b in enumerate(blocks):
        gen.fill(c, b)
    s_ref, U_ref = fp64_oracle(torch, blocks)
    torch.cuda.empty_cache()
    ctx = eb.Context(dev.index)
    pub, priv = eb.reference_seeds(0, P)
    dirty = [False]

    def restore():
        if dirty[0]:
            for c, b in enumerate(blocks):
                gen.fill(c, b)
        dirty[0] = True

    def check(o, k=None, regen=False):
        k = k or len(o[0])
        if regen:   # plain and mixed overwrite the blocks (Q, Q_p): the V reference needs X again
            for c, b in enumerate(blocks):
                gen.fill(c, b)
        a = {"sigma_rel_err_max": float(((o[0][:k] - s_ref[:k]).abs() / s_ref[:k]).max()), "sigma_count": len(o[0])}
        # the 50 signal vectors (relative gaps ~10%) one by one, and the noise
        # subspace as a whole (its values sit within ~2% of each other)
        sig = accuracy(torch, s_ref[:50], U_ref[:, :50], o[0][:50], o[1][:, :50], blocks,
                       [v[:50] for v in o[2]])
        a["signal_u_angle_max"] = sig["u_angle_max_all"]
        a["signal_v_angle_max"] = sig["v_angle_max_all"]
        if o[1].shape[1] > 50:
            a["noise_u_subspace_angle"] = float(torch.linalg.matrix_norm(U_ref[:, :50].T @ o[1][:, 50:], ord=2)
                                                .clamp(max=1.0).arcsin())
        return a

    out = {"workload": workload_name("c5"), "warmup": warmup, "steps": steps,
           "oracle": "cuSOLVER FP64 QR of every block, QR of the stacked R factors, SVD (stored X)"}
    # the exact-Gram mode leaves the blocks as they are: it runs first (full
    # spectrum, then the top 50) on the blocks as generated
    for pname in modes:
        dirty[0] = pname != "exact"
        r = time_fedsvd(torch, ctx, blocks, restore if pname != "exact" else (lambda: None), pub, priv,
                        PRECISION[pname], warmup, steps, dev, world,
                        check=lambda o, regen=(pname != "exact"): check(o, regen=regen))
        out[pname] = summarize(r, dgemm_peak, int8_peak)
        torch.cuda.empty_cache()
        if pname == "exact":
            r = time_fedsvd(torch, ctx, blocks, lambda: None, pub, priv, PRECISION["exact"], warmup, steps, dev,
                            world, top_k=50, check=lambda o: check(o, 50))
            out["exact_top50"] = summarize(r, dgemm_peak, int8_peak)
            torch.cuda.empty_cache()
    if "plain" in out and "exact" in out:
        out["speedup_exact_vs_plain"] = out["plain"]["value"] / out["exact"]["value"]
    ctx.close()
    del blocks, gen
    torch.cuda.empty_cache()
    return out


def roofline(prof, dgemm_peak, int8_peak=None):
    """Roofline of the dominant kernel class (by event time) of a run."""
    dom = max(prof, key=lambda k: prof[k][0])
    ms, nl, work = prof[dom]
    share = ms / sum(v[0] for v in prof.values())
    if dom == "dgemm":
        achieved = work / (ms * 1e-3) / 1e12
        return {"kernel": "dgemm_kernel (DMMA m8n8k4 FP64)", "bound": "tensor", "achieved": achieved,
                "peak": dgemm_peak, "unit": "TFLOP/s", "frac": achieved / dgemm_peak, "traffic": None,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 figure)",
                "launches": nl, "share": share}
    peaks = measured_peaks()
    if dom == "crt":   # int8 operations of the per-modulus tcgen05 GEMMs
        achieved = work / (ms * 1e-3) / 1e12
        if int8_peak:
            peak, src = int8_peak, ("cuBLAS int8 GEMM (torch._int_mm 8192^3) measured in this run; "
                                    "MEASURED_PEAKS.json has no int8 figure")
        else:
            peak, src = 2.0 * peaks["bf16_tflops"], "twice the measured dense bf16 burst (no int8 library GEMM)"
        return {"kernel": "crt_kernel (tcgen05 kind::i8, one GEMM per modulus)", "bound": "tensor",
                "achieved": achieved, "peak": peak, "unit": "TOP/s (int8)", "frac": achieved / peak,
                "traffic": CRT_TRAFFIC, "peak_source": src, "launches": nl, "share": share}
    achieved = work / (ms * 1e-3) / 1e9 if work else 0.0
    return {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": None, "launches": nl, "share": share}


# DRAM bytes (read + write) of one crt_kernel Gram launch at c2 (M = N = 1000,
# K = 500,000, 16 moduli), from the ncu capture at K = 100,000 scaled by K
# (the residue planes read once dominate; profiles/crt_kernel_gram_c2_100k.md).
CRT_TRAFFIC = {"bytes_per_launch": (1.677e9 + 71.5e6) * 5.0, "launch": "participant Gram, K = 500,000",
               "algorithmic_bytes": 16 * 1000 * 500_000 + 16 * 1000 * 1000 * 16,
               "source": "ncu dram__bytes_read.sum + dram__bytes_write.sum at K = 100,000, x5 (traffic grows with K)"}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return json.load(open(path))
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def workload_name(name, n=None):
    if name == "c3":
        rows = c3_rows(0)
        return (f"c3: 64 participants, rows {min(rows)}..{max(rows)} (sum {sum(rows)}) x 512 FP64, "
                f"entries N(0,1) x 10^U[-2,2] per participant")
    if name == "c4":
        n = n or C4_N
        return (f"c4: dense {n} x {n} FP64, {n // 16} clusters of 16 singular values at relative spacing 1e-10, "
                f"centres log-uniform in [1e-8, 1] (Householder bidiagonalisation, bisection + twisted vectors "
                f"for all {n} triplets, cluster refinement)")
    if name == "c5":
        return ("c5: 4 participants x 1000000 x 2000 FP64 (reference m=2000, local_n=1000000; 64 GB), rank 50 "
                "with singular values 1e3..10 plus N(0, 1e-3) noise")
    P, m, n0, _ = CONFIGS[name]
    n = n or n0
    return f"{name}: {P} participants x {n} x {m} FP64 (reference m={m}, local_n={n})"


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    P, m, n, spectrum = CONFIGS[args.config]
    if args.rows:
        n = args.rows
    workload = workload_name(args.config, n)
    cfg = {"workload": workload, "participants": P, "m": m, "local_n": n, "spectrum": spectrum,
           "mode": "svd_mode 1 (two-sided), opt_control 3, full spectrum",
           "l2": "inputs (%.1f GB) larger than L2; restored from a device copy before each step" % (
               (sum(c3_rows(0)) if args.config == "c3" else P * n) * m * 8 / 1e9),
           "parallelism": "replicas only" if args.gpus > 1 else "1 GPU"}
    if args.impl == "reference":
        if rank != 0:
            return
        # the reference's own CPU pipeline at full size on the same blocks the
        # GPU arm generates (written as its Client<c>.mat input files)
        td, P, m, ns = reference_data(args)
        vals, cores, ph = [], None, None
        try:
            for i in range(args.warmup + args.steps):
                v, ph, cores = reference_run(P, m, ns, td.name)
                if i >= args.warmup:
                    vals.append(v)
        finally:
            td.cleanup()
        val = statistics.median(vals)
        sample = (f"reference pipeline (oracle/_ref, its own sources, OpenBLAS for MKL) at full size "
                  f"(local_n={ns}), the same {spectrum} blocks as the GPU arm; the reference's own run() timer; "
                  f"median of {args.steps}")
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": val, "unit": "s", "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": val * 1e3,
                          "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic", "config": cfg,
                          "cpu_baseline": {"value": val, "unit": "s", "cores": cores, "kind": "reference",
                                           "sample": sample, "phases_s": ph},
                          "e2e": {"value": val, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    import torch
    if args.only:   # one of the other workloads alone (profiling and measurement runs)
        dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
        torch.cuda.set_device(dev)
        dp, ip = cublas_dgemm_peak(torch, dev), cublas_int8_peak(torch, dev)
        if args.only == "c4":
            e = extra_c4(rank, 1, 1, max(1, args.steps), n=args.c4_n)
        elif args.only == "c5":
            e = extra_c5(rank, 1, 1, max(1, args.steps), dp, ip)
        else:
            modes = ["plain", "mixed", "exact"] if args.only == "c3" else ["plain", "exact"]
            e = extra_blocks(args, rank, 1, args.only, modes, args.warmup, args.steps, dp, ip)
        print(json.dumps({args.only: e, "dgemm_peak_tflops": dp, "int8_peak_tops": ip}))
        return
    if world > 1:
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    res = run_ours(args, rank, world)
    extras = {}
    todo = [] if args.extras == "none" else (list(EXTRAS) if args.extras == "all" else args.extras.split(","))
    for name in todo:
        t0 = time.perf_counter()
        try:
            if name == "c1":
                e = extra_blocks(args, rank, world, "c1", ["plain", "exact"], 3, 10, res.get("dgemm_peak"),
                                 res.get("int8_peak"))
            elif name == "c3":
                e = extra_blocks(args, rank, world, "c3", ["plain", "mixed", "exact"], 2, 3,
                                 res.get("dgemm_peak"), res.get("int8_peak"))
            elif name == "c4":
                e = extra_c4(rank, world, 1, 2)
            elif name == "c5":
                e = extra_c5(rank, world, 1, 2, res.get("dgemm_peak"), res.get("int8_peak"))
            else:
                continue
        except Exception as ex:   # one workload's failure does not hide the others' numbers
            e = {"error": f"{type(ex).__name__}: {ex}"}
        e["wall_s"] = time.perf_counter() - t0
        extras[name] = e
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    runs = res["runs"]
    head = runs[res["head"]]
    prof = head["prof"]
    line = {"metric": METRIC, "value": head["sec"], "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["sec"] * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "precision": res["head"], "accuracy": head["acc"], "stage_ms": head["stage_ms"],
            "host_s_per_step": head["host_sec"], "gpu_launches": head["launches"],
            "roofline": roofline(prof, res["dgemm_peak"], res.get("int8_peak")),
            "batched_local_qr": (None if head["tuned"] is None else
                                 {"streams": head["tuned"][0], "panel_width": head["tuned"][1],
                                  "tuning_ms": head["tuned"][2], "graph": "captured on the 2nd call, replayed after"}),
            "kernel_classes": {k: {"ms": v[0], "launches": v[1]} for k, v in prof.items() if v[1]},
            "clocks": head["clocks"], "int8_peak_tops": res.get("int8_peak"), "dgemm_peak_tflops": res["dgemm_peak"]}
    if prof.get("sketch", (0, 0, 0))[1]:
        ms, nl, work = prof["sketch"]
        pk = measured_peaks()
        ach = work / 3.0 / (ms * 1e-3) / 1e12          # algorithmic 2 m N n per launch
        peak = pk["bf16_tflops"] / 3.0                   # BF16x3: three bf16 products per product
        line["roofline_sketch"] = {"kernel": "sketch_kernel (tcgen05 kind::f16 BF16x3, TMA, TMEM)",
                                   "bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                                   "frac": ach / peak, "launches": nl,
                                   "note": "algorithmic 2*m*N*n flops per launch against the measured bf16 "
                                           "burst peak / 3 (three bf16 products per FP64-equivalent product)"}
    for other, o in runs.items():   # the other precision modes, beside the headline one
        if other == res["head"]:
            continue
        line[other] = dict(summarize(o, res["dgemm_peak"], res.get("int8_peak"), head=True),
                           precision_mode=PRECISION[other])
    if "plain" in runs and res["head"] != "plain":
        line["speedup_vs_plain"] = runs["plain"]["sec"] / head["sec"]
    if "e2e" in res:
        line["e2e"] = res["e2e"]
    line.update(extras)
    if not args.no_cpu_baseline:
        # the reference's own pipeline at full size, once, on the same blocks
        try:
            td, Pr, mr, ns = reference_data(args)
            try:
                v, ph, cores = reference_run(Pr, mr, ns, td.name)
            finally:
                td.cleanup()
            line["cpu_baseline"] = {"value": v, "unit": "s", "cores": cores, "kind": "reference",
                                    "sample": f"one full-size run of the reference pipeline (oracle/_ref) on the "
                                              f"same blocks (local_n={ns}), its own run() timer",
                                    "phases_s": ph}
        except Exception as e:   # the checker build is missing on this machine
            line["cpu_baseline"] = {"value": None, "unit": "s", "cores": os.cpu_count(), "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
