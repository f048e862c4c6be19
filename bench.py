#!/usr/bin/env python3
"""Benchmark of the dense SPD path: FP64 Cholesky factor (dpotrf, lower) of one
n = 16384 SPD matrix A = G G^T / n + I (G i.i.d. uniform[-1, 1], seed 0) per step
on one B200, through the C ABI of libcucholesky.so (cuDpotrf).

One JSON line (rank 0):
  value   POTRF TFLOP/s (n^3/3 per step) with A resident in HBM; each step restores
          A from a pristine copy (a 2 GiB device copy, which also flushes L2) and
          factors it; the restore is inside the timed region.
  e2e     the same metric through the same C-ABI call with A in pinned HOST memory:
          host->device copy of A, cuDpotrf, device->host copy of the factor.
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
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--uplo", default="L")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--syrk", nargs=2, type=int, metavar=("M", "K"),
                    help="only the dominant kernel: two cuDsyrk(L, N) launches of order M, rank K "
                         "(warm-up + measured), for profiling")
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


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.syrk:
        run_syrk_only(*args.syrk)
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
    # of the factorization's first outer step, m = n - 512 rows, k = 256, timed with
    # CUDA events on the stream it is launched on
    bh = cc.BlasHandle()
    mk, kk = n - 512, 256
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
    # DRAM traffic per launch: 15.1 bytes per lower-triangle element of C, from the
    # ncu capture of the same kernel at m = 8192, k = 256 (profiles/), scaled by the
    # number of C elements (C's read + write dominate; the panel stays in L2)
    syrk_traffic = 15.1 * (float(mk) * (mk + 1) / 2)
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

    # end to end through the same C-ABI call with host buffers
    e2e = None
    if not args.no_e2e:
        hostA = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
        hostA.copy_(A0)
        hostF = torch.empty_like(hostA, pin_memory=True)
        dA = torch.empty_like(A0)
        torch.cuda.synchronize()
        for _ in range(1):
            dA.copy_(hostA, non_blocking=True)
            cc.call_potrf(h, "D", args.uplo, n, dA.data_ptr(), n)
            hostF.copy_(dA, non_blocking=True)
        torch.cuda.synchronize()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        k = max(1, min(args.steps, 3))
        s0.record()
        for _ in range(k):
            dA.copy_(hostA, non_blocking=True)
            rc, info = cc.call_potrf(h, "D", args.uplo, n, dA.data_ptr(), n)
            hostF.copy_(dA, non_blocking=True)
        s1.record()
        torch.cuda.synchronize()
        ems = s0.elapsed_time(s1) / k
        e2e = {"value": world * flops / (ems / 1e3) / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": n * n * 8, "d2h_bytes_per_step": n * n * 8, "ms_per_step": ems}
        del hostA, hostF, dA

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
                       "n": n, "uplo": args.uplo, "lda": n, "nb": 128,
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
