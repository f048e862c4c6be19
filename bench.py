#!/usr/bin/env python3
"""Benchmark of the dense SPD path: FP64 Cholesky factor (dpotrf, lower) of one
n = 16384 SPD matrix A = G G^T / n + I (G i.i.d. uniform[-1, 1], seed 0) per step
on one B200, through the C ABI of libcucholesky.so (cuDpotrf).

One JSON line (rank 0):
  value   POTRF TFLOP/s (n^3/3 per step) with A resident in HBM; each step restores
          A from a pristine copy (a 2 GiB device copy, which also flushes L2) and
          factors it; the restore is inside the timed region.
  e2e     the same metric through the reference's host-memory entry point
          cuMultiGPUDpotrf with A in pinned HOST memory: the call copies the lower
          triangle in, factors it, and copies each block column of the factor back
          behind the work that finishes it; timed by the host clock around the
          (synchronous) call, each step on a freshly restored host copy of A.
  roofline  achieved FP64 TFLOP/s of the factorisation (CUDA events around the
          potrf call only) against the FP64 tensor-core peak measured live on this
          GPU as the best cuBLAS DGEMM rate (8192^3), plus DRAM traffic (null here;
          the ncu capture under profiles/ gives it).
  cpu_baseline  the reference's own CPU dpotrf (oracle/_ref, compiled from its
          lapack/*.c over blas/*.c) on the host cores, on a bounded sample.

--impl reference times that reference CPU path alone (the reference has no
runnable GPU path: its kernels target sm_11/sm_13 and do not compile with nvcc
12.9).  Multi-GPU (torchrun, --gpus N): one independent matrix per rank
("replicas only": a single factorisation does not shard); value = total flops of
all ranks / max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cuda-cholesky_b200"))

N_DEFAULT = 16384
CPU_SAMPLE_N = 4096


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--n", type=int, default=None,
                    help="matrix order (default: 16384 for potrf, 32768 for mixed, 65536 for ozaki)")
    ap.add_argument("--uplo", default="L")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--kappa", default="0,1,2,3",
                    help="mixed workload: exponents k of D = diag(10^(k i/(n-1))), comma separated")
    ap.add_argument("--workload", default="potrf", choices=["potrf", "batched", "mixed", "ozaki"],
                    help="potrf: FP64 dpotrf n=16384 (default line); batched: 10,000 uneven SPD "
                         "kernel matrices, potrf + logdet + potri in one graph launch")
    ap.add_argument("--dtype", default="d", choices=["d", "s"], help="batched workload precision")
    ap.add_argument("--syrk", nargs=2, type=int, metavar=("M", "K"),
                    help="only the dominant kernel: two cuDsyrk(L, N) launches of order M, rank K "
                         "(warm-up + measured), for profiling")
    ap.add_argument("--syrk-lowp", nargs=3, metavar=("M", "K", "PREC"),
                    help="only the mixed factor's trailing update: two cuSsyrkLowp launches of order M, "
                         "rank K, PREC bf16 or tf32 (warm-up + measured), for profiling")
    return ap.parse_args()


def run_syrk_only(m: int, k: int) -> None:
    import torch
    import cucholesky as cc
    dev = torch.device("cuda", 0)
    bh = cc.BlasHandle()
    P = torch.randn(k, m, dtype=torch.float64, device=dev)     # column-major m x k
    C = torch.zeros(m, m, dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream()
    for _ in range(2):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        rc = cc.call_rankk(bh, "D", "L", "N", m, k, -1.0, P.data_ptr(), m, 1.0, C.data_ptr(), m, st.cuda_stream)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        print(json.dumps({"kernel": "cuDsyrk L,N", "m": m, "k": k, "rc": rc, "ms": ms,
                          "tflops": float(m) * (m + 1) * k / (ms / 1e3) / 1e12}), flush=True)
    bh.close()


def run_syrk_lowp_only(m: int, k: int, prec: str) -> None:
    import torch
    import cucholesky as cc
    dev = torch.device("cuda", 0)
    h = cc.Handle()
    p = cc.MIXED_BF16 if prec == "bf16" else cc.MIXED_TF32
    Q = (torch.rand((m, k), device=dev, dtype=torch.float32) * 2 - 1).to(
        torch.bfloat16 if prec == "bf16" else torch.float32)
    C = torch.zeros((m, m), device=dev, dtype=torch.float32)
    for _ in range(2):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        rc = cc.call_syrk_lowp(h, p, m, k, -1.0, Q.data_ptr(), k, C.data_ptr(), m)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        print(json.dumps({"kernel": f"cuSsyrkLowp {prec}", "m": m, "k": k, "rc": rc, "ms": ms,
                          "tflops": float(m) * (m + 1) * k / (ms / 1e3) / 1e12,
                          "c_gbs": float(m) * (m + 1) / 2 * 8 / (ms / 1e3) / 1e9}), flush=True)
    h.close()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------------------------
# CPU path of the reference (oracle/_ref) -- the baseline arm and cpu_baseline key
# ---------------------------------------------------------------------------------
def cpu_reference_rate(n: int, reps: int):
    """GFLOP/s of the reference's CPU dpotrf (lower) on the seeded SPD matrix of
    order n, all host cores.  Returns (tflops, cores, kind, seconds list)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from cucholesky import matgen
    kind = "reference" if O.available("reference") else "port"
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    A = matgen.spd("d", n, seed=0)
    times = []
    for _ in range(reps):
        F = A.copy(order="F")
        t0 = time.perf_counter()
        info = O.potrf("d", "L", F, impl=kind)
        times.append(time.perf_counter() - t0)
        assert info == 0
    best = min(times)
    return n ** 3 / 3 / best / 1e12, cores, kind, times


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    n = min(args.n, CPU_SAMPLE_N)
    rate, cores, kind, times = cpu_reference_rate(n, args.steps + args.warmup)
    timed = times[args.warmup:] or times
    ms = statistics.mean(timed) * 1e3
    v = n ** 3 / 3 / (ms / 1e3) / 1e12
    line = {
        "impl": "reference",
        "metric": "dpotrf_tflops", "value": v, "unit": "TFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"dpotrf lower FP64 n={args.n} (sample n={n}, reference CPU path)",
                   "n": args.n, "uplo": "L", "lda": args.n, "sample_n": n},
        "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": cores, "kind": kind,
                         "sample": f"dpotrf lower n={n}, {len(timed)} timed reps on the seeded SPD matrix"},
        "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------------
def fp64_peak_tflops(torch, dev):
    """FP64 dense peak on this GPU, measured live: best cuBLAS DGEMM 8192^3."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(4):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2 * n ** 3 / (best / 1e3) / 1e12


def make_spd_device(torch, n, seed, dev):
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    G = torch.rand(n, n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    A = G @ G.T
    A.div_(n)
    A.diagonal().add_(1.0)
    del G
    return A          # symmetric, so row/column-major are the same bytes


def run_batched(args) -> None:
    """10,000 squared-exponential kernel matrices K_ij = exp(-|x_i - x_j|^2 / (2 * 0.3^2))
    + 1e-4 delta_ij on n_i ~ U{8..512} points x ~ U[0,1]^3 (seed 0): factor, log det
    and inverse of every matrix in one graph launch of a batched plan, against
    looping the plain per-matrix calls (cu?potrf, cu?logdet, cu?potri) on a seeded
    sample of 200 matrices, extrapolated to the whole batch by sum n^3."""
    import numpy as np
    import torch
    import cucholesky as cc
    from cucholesky import shard
    rank, world, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    pg = None
    if world > 1:
        # the batch shards by matrix (cost-balanced), no exchange in the data path
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
        pg = dist
    p = args.dtype
    tdt = torch.float64 if p == "d" else torch.float32
    B = 10000
    rng = np.random.default_rng(0)
    sizes_all = rng.integers(8, 513, B).tolist()
    mine = shard.partition_by_cost(sizes_all, world)[rank] if world > 1 else list(range(B))
    sizes = [sizes_all[i] for i in mine]
    off, t = [], 0
    for n in sizes:
        off.append(t)
        t += n * n
    buf0 = torch.empty(max(t, 1), dtype=tdt, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    pos = {b: q for q, b in enumerate(mine)}
    for b, n in enumerate(sizes_all):          # every rank draws the same points in order
        x = torch.rand(n, 3, dtype=torch.float64, device=dev, generator=g)
        if b not in pos:
            continue
        o = off[pos[b]]
        K = torch.exp(-torch.cdist(x, x).pow(2) / (2 * 0.3 ** 2)) + 1e-4 * torch.eye(n, dtype=torch.float64, device=dev)
        buf0[o:o + n * n] = K.to(tdt).reshape(-1)     # symmetric: row- and column-major agree
    buf = buf0.clone()
    h = cc.Handle()
    t0 = time.perf_counter()
    plan = cc.BatchedPlan(h, buf, sizes, off, flags=7, nb=0)
    plan_s = time.perf_counter() - t0
    flops = float(sum(n ** 3 for n in sizes_all))    # n^3/3 (potrf) + 2n^3/3 (potri), whole batch
    for _ in range(args.warmup):
        buf.copy_(buf0)
        plan.run()
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        buf.copy_(buf0)
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        plan.run()
        e1.record()
        torch.cuda.synchronize()
        ms_r = e0.elapsed_time(e1)
        if pg is not None:                           # the step time is the slowest rank's
            tms = torch.tensor([ms_r], dtype=torch.float64, device=dev)
            pg.all_reduce(tms, op=pg.ReduceOp.MAX)
            ms_r = float(tms.item())
        times.append(ms_r)
    info, ld = plan.results()
    if pg is not None:                               # the one collective: gather the results
        info_all, ld_all = shard.gather_results(mine, info, ld, B, device=dev)
        n_failed = int((info_all != 0).sum().item())
    else:
        n_failed = sum(1 for i in info if i != 0)
    ms = statistics.mean(times)
    if rank != 0:
        plan.close()
        h.close()
        if pg is not None:
            pg.destroy_process_group()
        return
    B_local = len(sizes)
    # accuracy on a sample: inverse residual and log det against FP64 numpy
    chk = rng.choice(B_local, min(20, B_local), replace=False)
    host = buf.cpu().numpy()
    hres = buf0.cpu().numpy()
    worst_res = worst_ld = 0.0
    for b in chk:
        n, o = sizes[b], off[b]
        A = hres[o:o + n * n].reshape(n, n).astype(np.float64)
        X = np.tril(host[o:o + n * n].reshape(n, n, order="F").astype(np.float64))
        X = X + np.tril(X, -1).T
        kappa = np.linalg.cond(A)
        eps = np.finfo(np.float64 if p == "d" else np.float32).eps
        worst_res = max(worst_res, float(np.linalg.norm(np.eye(n) - A @ X) / (n * kappa * float(eps))))
        ref = float(np.linalg.slogdet(A)[1])
        worst_ld = max(worst_ld, float(abs(ld[b] - ref) / (n * float(eps) * max(1.0, abs(ref)))))
    # the same work as a loop of plain per-matrix calls, on a sample
    sample = rng.choice(B_local, min(200, B_local), replace=False)
    P = p.upper()
    # untimed warm-up of the plain calls (first launches load their kernels)
    for b in sample[:8]:
        n, o = sizes[b], off[b]
        ptr = buf.data_ptr() + o * buf.element_size()
        buf[o:o + n * n].copy_(buf0[o:o + n * n])
        cc.call_potrf(h, P, "L", n, ptr, n)
        cc.call_logdet(h, P, ptr, n + 1, n)
        cc.call_potri(h, P, "L", n, ptr, n)
    torch.cuda.synchronize()
    loop_ms = 0.0
    for b in sample:
        n, o = sizes[b], off[b]
        buf[o:o + n * n].copy_(buf0[o:o + n * n])
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        ptr = buf.data_ptr() + o * buf.element_size()
        e0.record()
        cc.call_potrf(h, P, "L", n, ptr, n)
        cc.call_logdet(h, P, ptr, n + 1, n)
        cc.call_potri(h, P, "L", n, ptr, n)
        e1.record()
        torch.cuda.synchronize()
        loop_ms += e0.elapsed_time(e1)
    frac = sum(sizes[b] ** 3 for b in sample) / flops
    loop_total_ms = loop_ms / frac
    line = {
        "metric": "batched_potrf_logdet_potri_matrices_per_s", "value": B / (ms / 1e3), "unit": "matrices/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "f64" if p == "d" else "f32",
        "data": "synthetic",
        "config": {"workload": "10,000 squared-exponential kernel matrices, n_i ~ U{8..512}, lower",
                   "batch": B, "sum_n3": flops, "graph_launches_per_step": 1, "nb": plan.nb,
                   "parallelism": f"sharded by cost over {world} GPUs" if world > 1 else "single"},
        "gflops": flops / (ms / 1e3) / 1e9,
        "loop_of_plain_calls_ms_extrapolated": loop_total_ms,
        "speedup_vs_loop": loop_total_ms / ms,
        "loop_sample": "200 matrices (seeded), cu?potrf + cu?logdet + cu?potri each, extrapolated by sum n^3",
        "failed_matrices": n_failed,
        "worst_inverse_residual_sampled": worst_res, "worst_logdet_rel_err_n_eps_sampled": worst_ld,
        "plan_build_s": plan_s,
    }
    print(json.dumps(line), flush=True)
    plan.close()
    h.close()
    if pg is not None:
        pg.destroy_process_group()


def run_mixed(args) -> None:
    """Mixed-precision refined SPD solve against the plain FP64 solve on the same GPU,
    n = 32768, 16 right-hand sides ~ N(0, 1): A = D (G G^T / n + 1e-3 I) D with
    G ~ N(0, 1) and D = diag(10^(k i / (n - 1))) for each k of --kappa (kappa ~1e3 to
    ~1e9).  FP64 arm: cuDpotrf + cuDpotrs on a restored copy of A.  Mixed arm, BF16
    and TF32 trailing updates: cuDcholMixedRefactor (scaling, |A|_inf, low-precision
    factor) + cuDcholMixedSolve (FP64 refinement to sqrt(n) eps).  Backward errors
    are recomputed here in FP64 (torch) for both arms."""
    import torch
    import cucholesky as cc
    from cucholesky import matgen
    dev = torch.device("cuda", 0)
    n = args.n if args.n is not None else 32768
    nrhs = 16
    ks = [float(k) for k in args.kappa.split(",")]
    h = cc.Handle()
    cases = []

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    for k in ks:
        A = matgen.scaled_spd_device(n, k, seed=int(k), device=dev)
        g = torch.Generator(device=dev)
        g.manual_seed(100 + int(k))
        B = torch.randn((nrhs, n), generator=g, device=dev, dtype=torch.float64)   # column-major n x 16
        anorm = A.abs().sum(dim=1).max().item()

        def berr(X):
            R = B - X @ A
            return float(max(R[c].abs().max().item() / (anorm * X[c].abs().max().item() + B[c].abs().max().item())
                             for c in range(nrhs)))

        # FP64: dpotrf + dpotrs
        Aw = torch.empty_like(A)
        X64 = torch.empty_like(B)
        t64 = []
        for it in range(args.warmup + args.steps):
            Aw.copy_(A)
            X64.copy_(B)

            def fp64():
                rc, info = cc.call_potrf(h, "D", "L", n, Aw.data_ptr(), n)
                assert rc == 0 and info == 0, (rc, info)
                rc, info = cc.call_potrs(h, "D", "L", n, nrhs, Aw.data_ptr(), n, X64.data_ptr(), n)
                assert rc == 0 and info == 0
            ms, _ = timed(fp64)
            if it >= args.warmup:
                t64.append(ms)
        b64 = berr(X64)
        del Aw
        torch.cuda.empty_cache()
        for prec, pname in ((cc.MIXED_TF32, "tf32"), (cc.MIXED_BF16, "bf16")):
            X = torch.zeros_like(B)
            plan = cc.MixedPlan(h, "L", n, A.data_ptr(), n, prec)
            tf, ts, iters = [], [], []
            res = (0, 0.0)
            for it in range(args.warmup + args.steps):
                msf, info = timed(plan.refactor)
                assert info == 0, info
                mss, res = timed(lambda: plan.solve(nrhs, B.data_ptr(), n, X.data_ptr(), n))
                if it >= args.warmup:
                    tf.append(msf)
                    ts.append(mss)
                    iters.append(res[0])
            shift = plan.factor()[4]
            plan.close()
            bm = berr(X)
            fwd = float((X - X64).abs().max().item() / X64.abs().max().item())
            t_mixed = statistics.mean(tf) + statistics.mean(ts)
            cases.append({
                "k": k, "precision": pname, "fp64_ms": statistics.mean(t64), "mixed_ms": t_mixed,
                "factor_ms": statistics.mean(tf), "refine_ms": statistics.mean(ts), "iterations": iters[-1],
                "speedup": statistics.mean(t64) / t_mixed, "berr_mixed": bm, "berr_fp64": b64,
                "berr_bound_10_n_eps": 10 * n * 2.0 ** -52, "rel_diff_vs_fp64_solution": fwd, "shift": shift,
                "effective_fp64_tflops_factor": n ** 3 / 3 / (statistics.mean(tf) / 1e3) / 1e12,
            })
            del X
        del A, B
        torch.cuda.empty_cache()
    # roofline of the dominant factor kernel: the tcgen05 trailing update at its largest
    # launch of this factorisation (m = n - 512 rows, k = 512), timed alone with CUDA events
    import json as _json
    peaks = {}
    try:
        peaks = _json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    bf16_peak = float(peaks.get("bf16_tflops", 1590.0))
    tf32_peak = bf16_peak / 2          # dense TF32 rate is half the BF16 rate on these tensor cores
    m, kq = n - 512, 512
    Cm = torch.rand((m, m), device=dev, dtype=torch.float32)
    upd = {}
    for prec, pname, qdt in ((cc.MIXED_TF32, "tf32", torch.float32), (cc.MIXED_BF16, "bf16", torch.bfloat16)):
        Qm = (torch.rand((m, kq), device=dev, dtype=torch.float32) * 2 - 1).to(qdt)
        for _ in range(3):
            cc.call_syrk_lowp(h, prec, m, kq, -1.0, Qm.data_ptr(), kq, Cm.data_ptr(), m)
        ts = []
        for _ in range(5):
            ms, _ = timed(lambda: cc.call_syrk_lowp(h, prec, m, kq, -1.0, Qm.data_ptr(), kq, Cm.data_ptr(), m))
            ts.append(ms)
        t = statistics.median(ts) / 1e3
        flop = float(m) * (m + 1) * kq          # lower triangle, 2 flop per multiply-add
        cbytes = float(m) * (m + 1) / 2 * 8     # C read + written once (FP32)
        upd[pname] = {"ms": t * 1e3, "tflops": flop / t / 1e12,
                      "tensor_frac": flop / t / 1e12 / (tf32_peak if pname == "tf32" else bf16_peak),
                      "c_gbs": cbytes / t / 1e9}
        del Qm
    del Cm
    torch.cuda.empty_cache()
    ok = [c for c in cases if c["k"] <= 2.0 and c["precision"] == "tf32"]
    value = min(c["speedup"] for c in ok) if ok else None
    line = {
        "metric": "mixed_refined_solve_speedup_vs_fp64_dpotrf_dpotrs", "value": value, "unit": "x",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": min(c["mixed_ms"] for c in ok) if ok else None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 (tf32/bf16 trailing updates)", "data": "synthetic",
        "config": {"workload": "SPD solve A = D (G G^T/n + 1e-3 I) D, G ~ N(0,1), D = diag(10^(k i/(n-1))), "
                               "16 rhs ~ N(0,1), lower", "n": n, "nrhs": nrhs, "k": ks,
                   "value": "min over k <= 2 (kappa <= ~4e7) of the TF32 speedup"},
        "cases": cases,
        "roofline": {"bound": "hbm", "achieved": upd["tf32"]["c_gbs"], "peak": hbm_peak, "unit": "GB/s",
                     "frac": upd["tf32"]["c_gbs"] / hbm_peak, "traffic": None,
                     "kernel": f"tc::update_kernel<tf32> (cuSsyrkLowp) m={m} k={kq}: C read+write, FP32",
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650 GB/s",
                     "tensor_tflops": upd["tf32"]["tflops"], "tensor_frac_of_tf32": upd["tf32"]["tensor_frac"],
                     "tf32_peak_tflops": tf32_peak, "bf16": upd["bf16"], "bf16_peak_tflops": bf16_peak},
    }
    print(json.dumps(line), flush=True)
    h.close()


def run_ozaki(args) -> None:
    """Large split-precision factor: dpotrf + dpotri of one FP64 SPD matrix
    A = G G^T / n + I (G uniform[-1, 1], seed 0), n = 65536 (34 GB) by default, with the
    trailing updates on the FP64 DMMA engine (cuDpotrf) and as the Ozaki-sliced INT8
    emulation (cuDpotrfOzaki, its default slice count: 7 at this order); the inverse (cuDpotri, the same native path
    for both) follows the Ozaki factor.  Errors are estimated with 4 Gaussian probes X
    (||E X||_F^2 / 4 estimates ||E||_F^2, O(n^2) work): the backward error
    ||A - L L^T||_F / (n eps ||A||_F) of each factor, and the inverse residual
    ||X - A (inv(A) X)||_F / (n eps ||A||_F ||inv(A) X||_F)."""
    import ctypes as C
    import torch
    import cucholesky as cc
    dev = torch.device("cuda", 0)
    n = args.n if args.n is not None else 65536
    eps = 2.0 ** -52
    h = cc.Handle()
    L = cc.lib()
    L.cuDpotrfOzaki.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_uint64, C.c_size_t, C.c_int,
                                C.POINTER(C.c_long)]
    L.cuDpotrfOzaki.restype = C.c_int

    slices = 7 if n >= 8192 else 8         # the library's default for this order

    def ozaki(ptr, nn, ld):
        info = C.c_long(0)
        rc = L.cuDpotrfOzaki(h.value, ord("L"), nn, ptr, ld, slices, C.byref(info))
        return rc, info.value

    # warm-up of both paths on a small matrix (kernel loading), untimed
    w = make_spd_device(torch, 2048, 1, dev)
    for f in (lambda t: cc.call_potrf(h, "D", "L", 2048, t.data_ptr(), 2048), lambda t: ozaki(t.data_ptr(), 2048, 2048)):
        t = w.clone()
        f(t)
    del w, t
    A0 = make_spd_device(torch, n, 0, dev)        # symmetric: row- and column-major agree
    anorm = torch.linalg.norm(A0).item()
    g = torch.Generator(device=dev)
    g.manual_seed(7)
    X = torch.randn((n, 4), generator=g, device=dev, dtype=torch.float64)

    def factor_error(T):
        # T: (n, n) tensor whose transpose is the column-major factor (L in its lower part)
        # L (L^T X) in row chunks of T = L^T (upper part of T): V = triu(T) X, W = triu(T)^T V
        V = torch.empty_like(X)
        ch = 4096
        for a in range(0, n, ch):
            b = min(n, a + ch)
            blk = torch.triu(T[a:b, a:], diagonal=0)
            V[a:b] = blk @ X[a:]
            del blk
        W = torch.zeros_like(X)
        for a in range(0, n, ch):
            b = min(n, a + ch)
            blk = torch.triu(T[a:b, a:], diagonal=0)
            W[a:] += blk.T @ V[a:b]
            del blk
        E = A0 @ X - W
        return float(torch.linalg.norm(E).item() / 2.0 / (n * eps * anorm))   # / sqrt(4 probes)

    Aw = torch.empty_like(A0)
    out = {}
    # each arm twice on a fresh copy of A; the first run of each also grows the
    # handle's workspace to its size, so the second is the one reported
    for name, call in (("native_dmma", lambda: cc.call_potrf(h, "D", "L", n, Aw.data_ptr(), n)),
                       ("ozaki_int8", lambda: ozaki(Aw.data_ptr(), n, n))):
        runs = []
        for _ in range(2):
            Aw.copy_(A0)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            rc, info = call()
            e1.record()
            torch.cuda.synchronize()
            runs.append(e0.elapsed_time(e1))
        ms = runs[-1]
        out[name] = {"potrf_ms": ms, "first_run_ms": runs[0], "tflops": n ** 3 / 3 / (ms / 1e3) / 1e12, "rc": rc,
                     "info": info, "backward_error_n_eps_probe": factor_error(Aw)}
    # the inverse from the Ozaki factor (native ?potri)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    rc, info = cc.call_potri(h, "D", "L", n, Aw.data_ptr(), n)
    e1.record()
    torch.cuda.synchronize()
    potri_ms = e0.elapsed_time(e1)
    # inverse residual: Y = inv(A) X from the lower triangle of Aw (symmetric), R = X - A Y
    ch = 4096
    Y = torch.zeros_like(X)
    for a in range(0, n, ch):
        b = min(n, a + ch)
        blk = torch.triu(Aw[a:b, a:], diagonal=0)   # rows a..b of the upper part of T = lower columns of inv(A)
        Y[a:b] += blk @ X[a:]
        strict = torch.triu(Aw[a:b, a:], diagonal=1)
        Y[a:] += strict.T @ X[a:b]
        del blk, strict
    R = X - A0 @ Y
    ynorm = torch.linalg.norm(Y).item()
    inv_res = float(torch.linalg.norm(R).item() / (anorm * ynorm * n * eps))
    line = {
        "metric": "ozaki_sliced_dpotrf_speedup_vs_native_dmma", "value": out["native_dmma"]["potrf_ms"] /
        out["ozaki_int8"]["potrf_ms"], "unit": "x", "n_gpus": 1, "steps": 1, "warmup": 1,
        "ms_per_step": out["ozaki_int8"]["potrf_ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (int8 slices)", "data": "synthetic",
        "config": {"workload": f"dpotrf + dpotri L FP64 n={n}, A=G*G^T/n+I, G~U[-1,1]", "n": n, "slices": slices},
        "arms": out, "potri_ms_after_ozaki": potri_ms, "potri_rc_info": [rc, info],
        "inverse_residual_probe_n_eps": inv_res,
        "error_note": "4 Gaussian probes: ||A X - L L^T X||_F / (2 n eps ||A||_F); ||X - A inv(A) X||_F / "
                      "(n eps ||A||_F ||inv(A) X||_F)",
    }
    print(json.dumps(line), flush=True)
    h.close()


def main():
    args = parse()
    if args.n is None and args.workload in ("potrf", "batched"):
        args.n = N_DEFAULT
    rank, world, local = dist_env()
    if args.syrk:
        run_syrk_only(*args.syrk)
        return
    if args.syrk_lowp:
        run_syrk_lowp_only(int(args.syrk_lowp[0]), int(args.syrk_lowp[1]), args.syrk_lowp[2])
        return
    if args.workload == "batched":
        if rank == 0:
            run_batched(args)
        return
    if args.workload == "mixed":
        if rank == 0:
            run_mixed(args)
        return
    if args.workload == "ozaki":
        if rank == 0:
            run_ozaki(args)
        return
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import torch
    import cucholesky as cc

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
        pg = dist

    n = args.n
    h = cc.Handle()
    lib = cc.lib()
    import ctypes as C
    peak = fp64_peak_tflops(torch, dev)

    A0 = make_spd_device(torch, n, seed=rank, dev=dev)
    A = torch.empty_like(A0)
    flops = n ** 3 / 3

    def launches():
        c = C.c_ulonglong(0)
        lib.cuLAPACKGetLaunchCount(h.value, C.byref(c))
        return c.value

    def step(ev=None):
        A.copy_(A0)
        if ev is not None:
            ev[0].record()
        rc, info = cc.call_potrf(h, "D", args.uplo, n, A.data_ptr(), n)
        if ev is not None:
            ev[1].record()
        if rc != 0 or info != 0:
            raise RuntimeError(f"cuDpotrf rc={rc} info={info}")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    l0 = launches()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for i in range(args.steps):
            step(evs[i])
        t1.record()
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
    nlaunch = launches() - l0

    # the dominant kernel alone: the trailing update (tensor-core SYRK) at the shape
    # of the factorization's first outer step, k = the outer block the tuning table
    # picks for this n (sub diagonal blocks of 128), m = n - k rows, timed with CUDA
    # events on the stream it is launched on
    bh = cc.BlasHandle()
    sub = C.c_int(0)
    lib.cuLAPACKGetPotrfBlocks.argtypes = [C.c_void_p, C.c_char, C.c_size_t, C.POINTER(C.c_int)]
    assert lib.cuLAPACKGetPotrfBlocks(h.value, b"D", n, C.byref(sub)) == 0
    kk = 128 * sub.value
    mk = n - kk
    Pk = torch.randn(kk, mk, dtype=torch.float64, device=dev)     # column-major mk x kk
    Ck = torch.zeros(mk, mk, dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream()
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(3)]
    cc.call_rankk(bh, "D", "L", "N", mk, kk, -1.0, Pk.data_ptr(), mk, 1.0, Ck.data_ptr(), mk, st.cuda_stream)
    for a, b in kev:
        a.record(st)
        rc = cc.call_rankk(bh, "D", "L", "N", mk, kk, -1.0, Pk.data_ptr(), mk, 1.0, Ck.data_ptr(), mk,
                           st.cuda_stream)
        b.record(st)
    torch.cuda.synchronize()
    syrk_ms = statistics.mean(a.elapsed_time(b) for a, b in kev)
    syrk_flops = float(mk) * (mk + 1) * kk          # lower triangle incl. diagonal
    syrk_tflops = syrk_flops / (syrk_ms / 1e3) / 1e12
    # DRAM traffic per launch, from the ncu captures of the same kernel at m = 8192
    # (profiles/): bytes per lower-triangle element of C (14.6 at k = 256, 16.05 at
    # k = 512; C's read + write) scaled by the number of C elements, plus the panel
    # read once (8 m k bytes; it stays in L2)
    syrk_traffic = (16.05 if kk >= 512 else 14.6) * (float(mk) * (mk + 1) / 2) + 8.0 * mk * kk
    del Pk, Ck
    bh.close()
    total_ms = t0.elapsed_time(t1)
    potrf_ms = [a.elapsed_time(b) for a, b in evs]
    if pg:
        t = torch.tensor([total_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * flops * args.steps / (total_ms / 1e3) / 1e12
    achieved = flops / (statistics.mean(potrf_ms) / 1e3) / 1e12

    # accuracy of the last factor: backward error from a sample of columns
    # ||A e_j - L (L^T e_j)|| over 64 columns, relative to n eps ||A e_j||
    idx = torch.linspace(0, n - 1, 64, device=dev).long()
    L = torch.tril(A.T if args.uplo == "L" else A)   # column-major lower == row-major upper
    Lt = L.T
    rhs = L @ Lt[:, idx]
    err = (A0[:, idx] - rhs).norm() / (n * torch.finfo(torch.float64).eps * A0[:, idx].norm())
    berr = float(err.item())
    del L, Lt, rhs

    # end to end through the host-memory entry point (cuMultiGPUDpotrf): A in pinned
    # host memory, restored before every call (untimed); the call returns when the
    # factor has landed in host memory, so the host clock around it is the e2e time
    e2e = None
    if not args.no_e2e:
        mg = cc.MultiGPU([local])
        hh = cc.HostHandle(mg)
        pristine = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
        pristine.copy_(A0)
        hostA = torch.empty_like(pristine, pin_memory=True)
        k = max(1, min(args.steps, 3))
        times, bytes_in, bytes_out, nl = [], [], [], []
        for it in range(1 + k):                    # the first call is untimed
            hostA.copy_(pristine)
            torch.cuda.synchronize()
            l0, i0, o0 = hh.stats()
            t_a = time.perf_counter()
            rc, info = cc.call_host(hh, "D", "potrf", args.uplo, n, hostA.data_ptr(), n)
            t_b = time.perf_counter()
            l1, i1, o1 = hh.stats()
            if rc != 0 or info != 0:
                raise RuntimeError(f"cuMultiGPUDpotrf rc={rc} info={info}")
            if it:
                times.append((t_b - t_a) * 1e3)
                bytes_in.append(i1 - i0)
                bytes_out.append(o1 - o0)
                nl.append(l1 - l0)
        ems = statistics.mean(times)
        if pg:
            t = torch.tensor([ems], device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {"value": world * flops / (ems / 1e3) / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": bytes_in[-1], "d2h_bytes_per_step": bytes_out[-1], "ms_per_step": ems,
               "entry_point": "cuMultiGPUDpotrf (host memory, include/lapack.h)", "steps": k,
               "gpu_launches_per_step": nl[-1], "clock": "host perf_counter around the synchronous call"}
        hh.close()
        mg.close()
        del pristine, hostA

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, cores, kind, times = cpu_reference_rate(CPU_SAMPLE_N, 2)
        cpu = {"value": rate, "unit": "TFLOP/s", "cores": cores, "kind": kind,
               "sample": f"dpotrf lower n={CPU_SAMPLE_N} (same generator), best of {len(times)}"}

    if rank == 0:
        line = {
            "metric": "dpotrf_tflops", "value": value, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"dpotrf {args.uplo} FP64 n={n} lda={n}, A=G*G^T/n+I, G~U[-1,1]",
                       "n": n, "uplo": args.uplo, "lda": n, "nb": 128, "outer_block": kk,
                       "l2": "each step restores A (2 GiB) from a pristine copy: inputs larger than L2",
                       "parallelism": "replicas" if world > 1 else "single"},
            "potrf_ms": statistics.mean(potrf_ms),
            "backward_error_sampled": berr,
            "roofline": {"bound": "tensor", "achieved": syrk_tflops, "peak": peak, "unit": "TFLOP/s",
                         "frac": syrk_tflops / peak, "traffic": syrk_traffic,
                         "kernel": f"dmma::gemm_kernel<0,0,0>: trailing-update SYRK (cuDsyrk L,N) m={mk} k={kk}",
                         "kernel_ms": syrk_ms, "algorithmic_flop": syrk_flops,
                         "algorithmic_bytes": 16.0 * (float(mk) * (mk + 1) / 2) + 8.0 * mk * kk,
                         "peak_source": "FP64 dense peak measured live: best cuBLAS DGEMM 8192^3 on this GPU"},
            "potrf_fraction_of_peak": achieved / peak,
            "potrf_achieved_tflops": achieved,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": nlaunch,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    h.close()
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
