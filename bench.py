"""Benchmark: decentralized SVD wall time on one B200 (per replica).

Workload (default): 2 participants, each holding a 500,000 x 1,000 FP64
block of X = U diag(s) V^T (U 10^6 x 1000 and V 1000 x 1000 Haar-random,
seeded; s geometric from 1 to 1e-6) — the reference's short-and-wide branch
with m = 1000 and local_n = 500,000.  One step is the whole pipeline
(local QR, masks, global QR, Ralha bidiagonalisation, bisection + twisted
vectors, back-transforms) on inputs resident in HBM; the 8 GB inputs are
larger than L2, and are restored from a pristine device copy before every
step (outside the timed events).

By default the three precision modes are timed: plain FP64 (mode 0, the
reference's Householder local QR), mixed (mode 1: BF16x3 tensor-core sketch +
FP64 Cholesky-QR refinement) and exact Gram (mode 2: the sketch as a
preconditioner of the exact Gram matrix, computed on the int8 tensor cores by
the Chinese remainder theorem, and products with the implicit Q made exact the
same way); the JSON value is mode 2, the other two sit beside it under
"plain" and "mixed".

Prints one JSON line (rank 0).  --impl reference times the reference's own
CPU implementation (oracle/_ref, built from the reference's sources) on a
bounded sample of the same workload.
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
}


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
    p.add_argument("--cpu-sample-rows", type=int, default=50_000)
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


def fp64_oracle(torch, blocks):
    """FP64 SVD of the stored X on the GPU (cuSOLVER Householder QR of every
    block, QR of the stacked R factors, SVD): the measurement's accuracy
    oracle, not part of the timed path.  X^T = Q R, so X = R^T Q^T."""
    Rs = [torch.linalg.qr(b.T, mode="r")[1] for b in blocks]
    R = torch.linalg.qr(torch.cat(Rs, dim=0), mode="r")[1]
    Ur, s, Vh = torch.linalg.svd(R.T)
    return s, Ur


def accuracy(torch, s_ref, U_ref, s, U):
    k = min(len(s), len(s_ref))
    rel = (s[:k] - s_ref[:k]).abs() / s_ref[:k]
    # gap-aware per-vector angles of the left singular vectors, sine form:
    # sin(angle) = || u - (u_ref . u) u_ref || (arccos of the cosine bottoms
    # out near 1.5e-8 in FP64)
    d = (U_ref[:, :k] * U[:, :k]).sum(dim=0)
    ang = torch.linalg.vector_norm(U[:, :k] - U_ref[:, :k] * d, dim=0).clamp(max=1.0).arcsin()
    gap = torch.full_like(s_ref[:k], float("inf"))
    gap[1:] = torch.minimum(gap[1:], s_ref[:k - 1] - s_ref[1:k])
    gap[:-1] = torch.minimum(gap[:-1], s_ref[:k - 1] - s_ref[1:k])
    well = (2.2e-16 * s_ref[0] / gap) <= 1e-10
    return {"sigma_rel_err_max": float(rel.max()), "sigma_count": int(len(s)),
            "u_angle_max_well_posed": float(ang[well].max()) if bool(well.any()) else None,
            "u_angle_max_all": float(ang.max())}


# ---------------------------------------------------------------- reference arm
def reference_run(P, m, n, seed=0, threads=None, workdir=None):
    """One run of the reference's own pipeline (oracle/_ref/ref_pipeline, P
    processes over loopback TCP; n is one local_n for all or a list).
    Returns (max run seconds over participants, per-phase seconds of
    participant 0, threads used)."""
    ns = list(n) if isinstance(n, (list, tuple)) else [n] * P
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_pipeline")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    cores = os.cpu_count() or 1
    threads = threads or max(1, cores // P)
    rng = np.random.default_rng(seed)
    with tempfile.TemporaryDirectory(dir=workdir) as td:
        for c in range(P):
            rng.standard_normal((m, ns[c])).tofile(os.path.join(td, f"Client{c}.mat"))
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS=str(threads))
        port = 20000 + (os.getpid() * 7 + int(time.time())) % 20000
        procs = []
        for c in range(P):
            od = os.path.join(td, f"o{c}")
            os.makedirs(od)
            procs.append(subprocess.Popen([exe, str(c), str(P), str(m), str(ns[c]), str(port), td, td, "0", "1", "-1", od],
                                          stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, env=env, cwd=td))
        for pr in procs:
            if pr.wait(timeout=1800) != 0:
                raise RuntimeError("reference participant failed")
        times = [list(map(float, open(os.path.join(td, f"o{c}", "time.txt")).read().split())) for c in range(P)]
    total = max(t[0] for t in times)
    ph = times[0]
    used = min(threads * P, cores)
    phases = dict(zip(("total", "local_qr", "global_qr", "apply_mask", "exchange", "bi_diag", "bsvd", "combine",
                       "comm"), ph))
    return total, phases, used


def reference_extrapolated(P, m, n_full, n_sample, steps=1, seed=0):
    """Reference time on a bounded sample (local_n = n_sample; lists allowed),
    extrapolated to local_n = n_full: the phases whose work grows with
    local_n (local QR, the V back-transform in combine) scale by the row
    ratio, the m-sized phases (masks, global QR, Ralha, bisection) are kept."""
    vals = []
    full = sum(n_full) if isinstance(n_full, (list, tuple)) else n_full * P
    samp = sum(n_sample) if isinstance(n_sample, (list, tuple)) else n_sample * P
    for i in range(steps):
        total, ph, cores = reference_run(P, m, n_sample, seed=seed + i)
        scale = full / samp
        grow = ph["local_qr"] + ph["combine"]
        vals.append(total + grow * (scale - 1.0))
    return statistics.median(vals), cores, ph


def sample_rows(args, P, n):
    """(full local_n, sampled local_n) for the CPU reference sample."""
    if args.config == "c3":
        full = c3_rows(0)
        return full, [max(3100, r // 20) for r in full]
    return n, min(args.cpu_sample_rows, n)


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


def max_over_ranks(torch, value, device, world):
    """The largest of every rank's value (a collective every rank calls in
    the same order): the job-level time of replicas timed independently."""
    if world <= 1:
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t)


def run_ours(args, rank, world):
    """Times the pipeline at each requested precision (plain FP64 first, then
    mixed); returns {precision: result} plus the end-to-end measurement of the
    headline precision."""
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
    s_ref, U_ref = fp64_oracle(torch, pristine)
    pub, priv = eb.reference_seeds(0, P)
    batched = sum(1 for b in pristine if b.shape[1] // m > 5) >= 8
    precisions = {"both": ["plain", "mixed"], "plain": ["plain"], "mixed": ["mixed"], "exact": ["exact"],
                  "all": ["plain", "mixed", "exact"]}[args.precision]
    out_all = {}
    for pname in precisions:
        prec = PRECISION[pname]
        tuned = ctx.fedsvd_tune(m, [b.shape[1] for b in pristine], precision=prec) if batched else None
        for _ in range(args.warmup):
            for b, p0 in zip(blocks, pristine):
                b.copy_(p0)
            torch.cuda.synchronize()
            out = ctx.fedsvd(blocks, pub, priv, precision=prec)
        acc = accuracy(torch, s_ref, U_ref, out[0], out[1])
        del out
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        l0 = ctx.launches()
        times = []
        stage = {}
        ctx.profile(True)
        with Clocks(dev.index) as clk:
            for _ in range(args.steps):
                for b, p0 in zip(blocks, pristine):
                    b.copy_(p0)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                out = ctx.fedsvd(blocks, pub, priv, precision=prec)      # synchronises before returning
                times.append(time.perf_counter() - t0)
                for kk, v in ctx.stage_ms().items():
                    stage[kk] = stage.get(kk, 0.0) + v / args.steps
                del out
        prof = ctx.profile_get()
        ctx.profile(False)
        launches = (ctx.launches() - l0) // args.steps
        torch.cuda.synchronize()
        # device time of a step = sum of its stage events (CUDA events on the stream)
        sec = max_over_ranks(torch, sum(stage.values()) / 1e3, dev, world)
        out_all[pname] = {"sec": sec, "host_sec": statistics.median(times), "stage_ms": stage, "acc": acc,
                          "tuned": tuned, "launches": launches, "prof": prof, "clocks": clk.summary()}
    res = {"runs": out_all, "head": precisions[-1]}
    if rank == 0:
        res["dgemm_peak"] = cublas_dgemm_peak(torch, dev)
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
    return res


def roofline(prof, dgemm_peak):
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
        peak = 2.0 * peaks["bf16_tflops"]
        return {"kernel": "crt_kernel (tcgen05 kind::i8, one GEMM per modulus)", "bound": "tensor",
                "achieved": achieved, "peak": peak, "unit": "TOP/s (int8)", "frac": achieved / peak, "traffic": None,
                "peak_source": "twice the measured dense bf16 burst (the tensor cores' 8-bit rate is twice their "
                               "16-bit rate); MEASURED_PEAKS.json has no int8 figure",
                "launches": nl, "share": share}
    achieved = work / (ms * 1e-3) / 1e9 if work else 0.0
    return {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": None, "launches": nl, "share": share}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return json.load(open(path))
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    P, m, n, spectrum = CONFIGS[args.config]
    if args.rows:
        n = args.rows
    if args.config == "c3":
        rows = c3_rows(0)
        workload = (f"c3: 64 participants, rows {min(rows)}..{max(rows)} (sum {sum(rows)}) x 512 FP64, "
                    f"entries N(0,1) x 10^U[-2,2] per participant")
    else:
        workload = f"{args.config}: {P} participants x {n} x {m} FP64 (reference m={m}, local_n={n})"
    cfg = {"workload": workload, "participants": P, "m": m, "local_n": n, "spectrum": spectrum,
           "mode": "svd_mode 1 (two-sided), opt_control 3, full spectrum",
           "l2": "inputs (%.1f GB) larger than L2; restored from a device copy before each step" % (
               (sum(c3_rows(0)) if args.config == "c3" else P * n) * m * 8 / 1e9),
           "parallelism": "replicas only" if args.gpus > 1 else "1 GPU"}
    if args.impl == "reference":
        if rank != 0:
            return
        nfull, ns = sample_rows(args, P, n)
        vals = []
        for i in range(args.warmup + args.steps):
            v, cores, ph = reference_extrapolated(P, m, nfull, ns, steps=1, seed=i)
            if i >= args.warmup:
                vals.append(v)
        val = statistics.median(vals)
        sample = (f"reference pipeline (oracle/_ref, its own sources) at local_n={ns}; local QR and "
                  f"back-transform phases scaled to the full row count")
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": val, "unit": "s", "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": val * 1e3,
                          "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic", "config": cfg,
                          "cpu_baseline": {"value": val, "unit": "s", "cores": cores, "kind": "reference",
                                           "sample": sample},
                          "e2e": {"value": val, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    if world > 1:
        import torch
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    res = run_ours(args, rank, world)
    if world > 1:
        import torch
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
            "roofline": roofline(prof, res["dgemm_peak"]),
            "batched_local_qr": (None if head["tuned"] is None else
                                 {"streams": head["tuned"][0], "panel_width": head["tuned"][1],
                                  "tuning_ms": head["tuned"][2], "graph": "captured on the 2nd call, replayed after"}),
            "kernel_classes": {k: {"ms": v[0], "launches": v[1]} for k, v in prof.items() if v[1]},
            "clocks": head["clocks"]}
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
        line[other] = {"value": o["sec"], "unit": "s", "precision_mode": PRECISION[other], "accuracy": o["acc"],
                       "stage_ms": o["stage_ms"], "gpu_launches": o["launches"],
                       "roofline": roofline(o["prof"], res["dgemm_peak"]),
                       "kernel_classes": {k: {"ms": v[0], "launches": v[1]} for k, v in o["prof"].items() if v[1]}}
    if "plain" in runs and res["head"] != "plain":
        line["speedup_vs_plain"] = runs["plain"]["sec"] / head["sec"]
    if "e2e" in res:
        line["e2e"] = res["e2e"]
    if not args.no_cpu_baseline:
        nfull, ns = sample_rows(args, P, n)
        try:
            v, cores, ph = reference_extrapolated(P, m, nfull, ns, steps=1)
            line["cpu_baseline"] = {"value": v, "unit": "s", "cores": cores, "kind": "reference",
                                    "sample": f"reference pipeline at local_n={ns}, local QR and back-transform "
                                              f"phases scaled to the full row count", "sample_phases_s": ph}
        except Exception as e:   # the checker build is missing on this machine
            line["cpu_baseline"] = {"value": None, "unit": "s", "cores": os.cpu_count(), "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
