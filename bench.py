#!/usr/bin/env python3
"""Benchmark of the dense SPD path on one B200, through the C ABI of libcucholesky.so.

Headline (the JSON line's metric / value / e2e): the plain FP64 drop-in, dpotrf
(lower) of one n = 16384 SPD matrix A = G G^T / n + I (G i.i.d. uniform[-1, 1],
torch Philox on the device, seed = rank) per step.

  value     POTRF TFLOP/s (n^3/3 per step) with A resident in HBM; each step restores
            A from a pristine copy (a 2 GiB device copy, which also flushes L2) and
            factors it (cuDpotrf); the restore is inside the timed region.
  e2e       the same metric through the reference's host-memory entry point
            cuMultiGPUDpotrf with A in pinned HOST memory: the call copies the lower
            triangle in, factors it, and copies each block column of the factor back
            behind the work that finishes it; host clock around the synchronous call.
  roofline  the dominant kernel (the trailing-update SYRK on the FP64 tensor cores,
            dmma::gemm_kernel) at the factorization's largest trailing update, timed
            with CUDA events on its stream, against the FP64 dense peak measured live
            (best cuBLAS DGEMM 8192^3, with the clocks seen during that probe); its
            DRAM traffic per launch is the ncu-measured bytes per lower-triangle element
            of C (dram__bytes_read.sum + dram__bytes_write.sum at m = 8192 on the
            64 x 64-tile kernel: 15.28 B at k = 512; 14.6 B at k = 256 on the earlier
            128 x 64-tile one) times the elements, plus the panel once.
  cpu_baseline  the reference's own CPU dpotrf (oracle/_ref, compiled from its
            lapack/*.c over blas/*.c, all host cores) on the GPU arm's own matrix at the
            same n = 16384: one untimed and two timed runs.

The same line carries the other targets of the path, each measured with fixed small
step counts (independent of --steps) and with its own roofline:
  potrf_n32768  dpotrf at n = 32768 (fraction of the FP64 peak, probe backward error)
  types         cuSpotrf / cuCpotrf / cuZpotrf (+ ?potri) at n = 16384 / 8192 / 8192
  mixed         the mixed-precision refined solve at n = 32768, kappa ~4e3 .. ~4e9,
                TF32 and BF16 trailing updates, against cuDpotrf + cuDpotrs
  batched       10,000 uneven SPD kernel matrices (n 8..512): potrf + logdet + potri in
                one graph launch, FP64 and FP32, against looping the plain calls
  ozaki         dpotrf + dpotri at n = 65536 with Ozaki-sliced INT8 trailing updates
                against the native FP64 tensor-core factor
(--no-extras leaves them out; --workload mixed|batched|ozaki prints one of them as its
own line.)

--impl reference times the reference's CPU dpotrf alone (the reference has no
runnable GPU path: its kernels target sm_11/sm_13 and do not compile with nvcc 12.9)
on the same matrix: each step factors a leading principal submatrix of it, of the
order that keeps the whole --steps/--warmup run within a few minutes (the full order
when that fits); the line says which.  Multi-GPU (torchrun, --gpus N): one
independent matrix per rank ("replicas only": a single factorization does not shard);
value = total flops of all ranks / max time over ranks.
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
import traceback

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cuda-cholesky_b200"))

N_DEFAULT = 16384
CPU_RATE_GUESS = 0.025e12      # reference CPU dpotrf on 16 host cores near n = 9000, flop/s (sizes the sample)
REF_ARM_BUDGET_S = 240.0       # whole --impl reference run


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
    ap.add_argument("--no-extras", action="store_true", help="only the headline dpotrf line")
    ap.add_argument("--extras", default="potrf_n32768,types,mixed,batched,ozaki",
                    help="comma-separated extras to add to the headline line")
    ap.add_argument("--kappa", default="0,1,2,3",
                    help="mixed workload: exponents k of D = diag(10^(k i/(n-1))), comma separated")
    ap.add_argument("--workload", default="potrf", choices=["potrf", "batched", "mixed", "ozaki"],
                    help="potrf: the default line; batched / mixed / ozaki: that target as its own line")
    ap.add_argument("--dtype", default="d", choices=["d", "s"], help="batched workload precision")
    ap.add_argument("--syrk", nargs=2, type=int, metavar=("M", "K"),
                    help="only the dominant kernel: two cu?syrk / cu?herk(L, N) launches of order M, "
                         "rank K (warm-up + measured), for profiling")
    ap.add_argument("--syrk-type", default="D", choices=["D", "Z"],
                    help="--syrk element type: D (cuDsyrk) or Z (cuZherk)")
    ap.add_argument("--single", nargs=2, metavar=("P", "N"),
                    help="only one cu<P>potrf of order N (P in S D C Z, --uplo), after one untimed call: "
                         "for profiling")
    ap.add_argument("--batch", type=int, default=10000, help="batched workload: number of matrices")
    ap.add_argument("--batched-nb", type=int, default=0,
                    help="batched workload: plan block size (0 tuned, 32 / 64 grouped graph, -1 persistent)")
    ap.add_argument("--syrk-lowp", nargs=3, metavar=("M", "K", "PREC"),
                    help="only the mixed factor's trailing update: two cuSsyrkLowp launches of order M, "
                         "rank K, PREC bf16 or tf32 (warm-up + measured), for profiling")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def timed(torch, fn, stream=None):
    """(ms, result) of fn() between CUDA events on `stream` (default: current)."""
    st = stream if stream is not None else torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    out = fn()
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), out


def guarded(name, fn):
    """Run one extra; a failure is recorded in the line instead of ending the run."""
    try:
        return fn()
    except Exception as exc:                       # noqa: BLE001 - reported, not hidden
        traceback.print_exc()
        return {"error": f"{type(exc).__name__}: {exc}"}
    finally:
        try:
            import torch
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
        except Exception:                           # noqa: BLE001
            pass


# ---------------------------------------------------------------------------------
# clocks during a timed region
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
# CPU path of the reference (oracle/_ref): the baseline arm and the cpu_baseline key
# ---------------------------------------------------------------------------------
def cpu_reference_times(A_host, n_s: int, reps: int):
    """Seconds of the reference's CPU dpotrf (lower) on the leading n_s x n_s block
    of the column-major host matrix A_host, `reps` runs, all host cores.  Returns
    (times, cores, kind)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    kind = "reference" if O.available("reference") else "port"
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    times = []
    for _ in range(reps):
        F = np.array(A_host[:n_s, :n_s], order="F", copy=True)
        t0 = time.perf_counter()
        info = O.potrf("d", "L", F, impl=kind)
        times.append(time.perf_counter() - t0)
        if info != 0:
            raise RuntimeError(f"reference dpotrf info={info}")
        del F
    return times, cores, kind


def host_matrix(torch, n, seed, dev):
    """The GPU arm's input matrix (device generator), copied to host memory in
    column-major order."""
    import numpy as np
    A = make_spd_device(torch, n, seed, dev)
    H = np.asfortranarray(A.cpu().numpy().T)       # symmetric: the same bytes
    del A
    torch.cuda.empty_cache()
    return H


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    import torch
    n = args.n
    reps = args.steps + args.warmup
    per_step = REF_ARM_BUDGET_S / max(reps, 1)
    n_s = min(n, int((3.0 * CPU_RATE_GUESS * per_step) ** (1.0 / 3.0)) // 512 * 512)
    n_s = max(n_s, 512)
    dev = torch.device("cuda", 0) if torch.cuda.is_available() else None
    if dev is not None:
        A = host_matrix(torch, n, 0, dev)
    else:                                            # same family, host generator
        from cucholesky import matgen
        A = matgen.spd("d", n, seed=0)
    times, cores, kind = cpu_reference_times(A, n_s, reps)
    timed_s = times[args.warmup:] or times
    ms = statistics.mean(timed_s) * 1e3
    v = n_s ** 3 / 3 / (ms / 1e3) / 1e12
    sample = (f"dpotrf lower on the leading {n_s} x {n_s} block of the n={n} matrix of the GPU arm "
              f"(seed 0), {len(timed_s)} timed + {args.warmup} untimed runs, {cores} threads"
              if n_s < n else f"dpotrf lower n={n} on the GPU arm's matrix (seed 0), {len(timed_s)} timed runs")
    line = {
        "impl": "reference",
        "metric": "dpotrf_tflops", "value": v, "unit": "TFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": headline_config(n, args.uplo, world),
        "sample": sample, "sample_n": n_s,
        "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------
# GPU helpers
# ---------------------------------------------------------------------------------
def fp64_peak_tflops(torch, dev, index):
    """FP64 dense peak on this GPU, measured live: best cuBLAS DGEMM 8192^3, with the
    clocks sampled while it ran."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 1e30
    with ClockSampler(index) as clk:
        for _ in range(6):
            ms, _ = timed(torch, lambda: a @ b)
            best = min(best, ms)
    del a, b
    torch.cuda.empty_cache()
    return 2 * n ** 3 / (best / 1e3) / 1e12, clk.summary()


def make_spd_device(torch, n, seed, dev):
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    G = torch.rand(n, n, dtype=torch.float64, device=dev, generator=g) * 2 - 1
    A = G @ G.T
    A.div_(n)
    A.diagonal().add_(1.0)
    del G
    return A          # symmetric, so row/column-major are the same bytes


def headline_config(n, uplo, world):
    return {"workload": f"dpotrf {uplo} FP64 n={n} lda={n}, A=G*G^T/n+I, G~U[-1,1]",
            "n": n, "uplo": uplo, "lda": n, "nb": 128,
            "l2": "each step restores A (2 GiB) from a pristine copy: inputs larger than L2",
            "parallelism": "replicas" if world > 1 else "single"}


def tuned_outer_block(cc, h, prefix, n):
    import ctypes as C
    lib = cc.lib()
    lib.cuLAPACKGetPotrfBlocks.argtypes = [C.c_void_p, C.c_char, C.c_size_t, C.POINTER(C.c_int)]
    sub = C.c_int(0)
    assert lib.cuLAPACKGetPotrfBlocks(h.value, prefix.encode(), n, C.byref(sub)) == 0
    return sub.value * (64 if prefix == "Z" else 128)


def syrk_roofline(torch, cc, prefix, m, k, peak, reps=3):
    """The trailing-update kernel alone (cu?syrk / cu?herk, lower, N) at order m and
    rank k, CUDA events on its stream: (ms, achieved TFLOP/s, algorithmic flop)."""
    dt = {"D": torch.float64, "Z": torch.complex128}[prefix]
    bh = cc.BlasHandle()
    P = torch.randn(k, m, dtype=dt, device="cuda")     # column-major m x k
    Cm = torch.zeros(m, m, dtype=dt, device="cuda")
    st = torch.cuda.current_stream()
    call = lambda: cc.call_rankk(bh, prefix, "L", "N", m, k, -1.0, P.data_ptr(), m, 1.0, Cm.data_ptr(), m,
                                 st.cuda_stream)
    call()
    ts = [timed(torch, call, st)[0] for _ in range(reps)]
    bh.close()
    del P, Cm
    torch.cuda.empty_cache()
    ms = statistics.mean(ts)
    flop = float(m) * (m + 1) * k * (4 if prefix == "Z" else 1)
    return ms, flop / (ms / 1e3) / 1e12, flop


# ---------------------------------------------------------------------------------
# extras: the other targets of the path
# ---------------------------------------------------------------------------------
def extra_potrf_large(torch, cc, h, peak, n=32768):
    """dpotrf (lower) at n = 32768: best of 2 timed runs after one untimed one."""
    from cucholesky import matgen
    A0 = make_spd_device(torch, n, 0, "cuda")
    A = torch.empty_like(A0)
    ts = []
    for it in range(3):
        A.copy_(A0)
        ms, (rc, info) = timed(torch, lambda: cc.call_potrf(h, "D", "L", n, A.data_ptr(), n))
        assert rc == 0 and info == 0, (rc, info)
        if it:
            ts.append(ms)
    L = matgen.factor_of(A, "L")
    del A
    torch.cuda.empty_cache()
    be = matgen.probe_backward_error(A0, L, "d")
    del L, A0
    torch.cuda.empty_cache()
    ms = min(ts)
    tf = n ** 3 / 3 / (ms / 1e3) / 1e12
    k = tuned_outer_block(cc, h, "D", n)
    kms, ktf, kflop = syrk_roofline(torch, cc, "D", n - k, k, peak)
    return {"n": n, "potrf_ms": ms, "tflops": tf, "fraction_of_fp64_peak": tf / peak, "outer_block": k,
            "backward_error_n_eps_probe": be, "bound_10": be <= 10,
            "roofline": {"bound": "tensor", "achieved": ktf, "peak": peak, "unit": "TFLOP/s", "frac": ktf / peak,
                         "kernel": f"dmma::gemm_kernel<0,0,0,2> SYRK m={n - k} k={k}", "kernel_ms": kms,
                         "algorithmic_flop": kflop}}


def extra_types(torch, cc, h, peak):
    """cu?potrf + cu?potri (lower) of the C2 inputs of the other three types, with the
    probe backward error of the factor and the inverse residual."""
    from cucholesky import matgen
    out = {}
    for p, n in (("s", 16384), ("c", 8192), ("z", 8192)):
        A0 = matgen.spd_device(p, n, seed=0).to(matgen.torch_dtype(p))
        A = torch.empty_like(A0)
        P = p.upper()
        mult = 4 if p in "cz" else 1
        ts = []
        for it in range(3):
            A.copy_(A0)
            ms, (rc, info) = timed(torch, lambda: cc.call_potrf(h, P, "L", n, A.data_ptr(), n))
            assert rc == 0 and info == 0, (p, rc, info)
            if it:
                ts.append(ms)
        Aexact = matgen.hermitian_of(A0, "L")
        be = matgen.probe_backward_error(Aexact, matgen.factor_of(A, "L"), p)
        ms_i, (rc, info) = timed(torch, lambda: cc.call_potri(h, P, "L", n, A.data_ptr(), n))
        assert rc == 0 and info == 0
        ir = matgen.probe_inverse_residual(Aexact, matgen.hermitian_of(A, "L"), p)
        del A, A0, Aexact
        torch.cuda.empty_cache()
        ms = min(ts)
        tf = mult * n ** 3 / 3 / (ms / 1e3) / 1e12
        rec = {"n": n, "potrf_ms": ms, "potrf_tflops": tf, "potri_ms": ms_i,
               "potri_tflops": mult * 2 * n ** 3 / 3 / (ms_i / 1e3) / 1e12,
               "backward_error_n_eps_probe": be, "inverse_residual_probe": ir,
               "flop_convention": "real-flop equivalents (x4 for complex)"}
        if p == "z":
            k = tuned_outer_block(cc, h, "Z", n)
            kms, ktf, kflop = syrk_roofline(torch, cc, "Z", n - k, k, peak)
            rec["potrf_fraction_of_fp64_peak"] = tf / peak
            rec["roofline"] = {"bound": "tensor", "achieved": ktf, "peak": peak, "unit": "TFLOP/s",
                               "frac": ktf / peak, "kernel": f"zmma::gemm_kernel<0,0,0> HERK m={n - k} k={k}",
                               "kernel_ms": kms, "algorithmic_flop": kflop}
        out[p] = rec
    return out


def mixed_result(torch, cc, h, n, ks, warmup, steps):
    """Mixed-precision refined SPD solve against the plain FP64 solve on the same GPU,
    n = 32768, 16 right-hand sides ~ N(0, 1): A = D (G G^T / n + 1e-3 I) D with
    G ~ N(0, 1) and D = diag(10^(k i / (n - 1))) for each k (kappa ~1e3 to ~1e9).
    FP64 arm: cuDpotrf + cuDpotrs on a restored copy of A.  Mixed arm, BF16 and TF32
    trailing updates: cuDcholMixedRefactor (scaling, low-precision factor) +
    cuDcholMixedSolve (FP64 refinement to sqrt(n) eps).  Backward errors are
    recomputed here in FP64 (torch) for both arms."""
    from cucholesky import matgen
    dev = torch.device("cuda", 0)
    nrhs = 16
    cases = []
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

        Aw = torch.empty_like(A)
        X64 = torch.empty_like(B)
        t64 = []
        for it in range(warmup + steps):
            Aw.copy_(A)
            X64.copy_(B)

            def fp64():
                rc, info = cc.call_potrf(h, "D", "L", n, Aw.data_ptr(), n)
                assert rc == 0 and info == 0, (rc, info)
                rc, info = cc.call_potrs(h, "D", "L", n, nrhs, Aw.data_ptr(), n, X64.data_ptr(), n)
                assert rc == 0 and info == 0
            ms, _ = timed(torch, fp64)
            if it >= warmup:
                t64.append(ms)
        b64 = berr(X64)
        del Aw
        torch.cuda.empty_cache()
        for prec, pname in ((cc.MIXED_TF32, "tf32"), (cc.MIXED_BF16, "bf16")):
            X = torch.zeros_like(B)
            plan = cc.MixedPlan(h, "L", n, A.data_ptr(), n, prec)
            tf, ts, iters = [], [], []
            for it in range(warmup + steps):
                msf, info = timed(torch, plan.refactor)
                assert info == 0, info
                mss, res = timed(torch, lambda: plan.solve(nrhs, B.data_ptr(), n, X.data_ptr(), n))
                if it >= warmup:
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
                "berr_bound_10_n_eps": 10 * n * 2.0 ** -52, "within_bound": bm <= 10 * n * 2.0 ** -52,
                "rel_diff_vs_fp64_solution": fwd, "shift": shift,
                "effective_fp64_tflops_factor": n ** 3 / 3 / (statistics.mean(tf) / 1e3) / 1e12,
            })
            del X
        del A, B
        torch.cuda.empty_cache()
    # roofline of the dominant factor kernel: the tcgen05 trailing update at its largest
    # launch of this factorization (m = n - 512 rows, k = 512), timed alone
    peaks = load_peaks()
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    bf16_peak = float(peaks.get("bf16_tflops", 1590.0))
    tf32_peak = bf16_peak / 2          # the dense TF32 rate of these tensor cores is half the BF16 rate
    m, kq = n - 512, 512
    Cm = torch.rand((m, m), device=dev, dtype=torch.float32)
    upd = {}
    for prec, pname, qdt in ((cc.MIXED_TF32, "tf32", torch.float32), (cc.MIXED_BF16, "bf16", torch.bfloat16)):
        Qm = (torch.rand((m, kq), device=dev, dtype=torch.float32) * 2 - 1).to(qdt)
        for _ in range(3):
            cc.call_syrk_lowp(h, prec, m, kq, -1.0, Qm.data_ptr(), kq, Cm.data_ptr(), m)
        ts = [timed(torch, lambda: cc.call_syrk_lowp(h, prec, m, kq, -1.0, Qm.data_ptr(), kq, Cm.data_ptr(), m))[0]
              for _ in range(5)]
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
    return {
        "metric": "mixed_refined_solve_speedup_vs_fp64_dpotrf_dpotrs",
        "value": min(c["speedup"] for c in ok) if ok else None, "unit": "x",
        "value_definition": "min over k <= 2 (kappa <= ~4e7) of the TF32 speedup",
        "n": n, "nrhs": nrhs, "k": list(ks), "steps": steps, "warmup": warmup,
        "workload": "SPD solve A = D (G G^T/n + 1e-3 I) D, G ~ N(0,1), D = diag(10^(k i/(n-1))), 16 rhs, lower",
        "cases": cases,
        "roofline": {"bound": "hbm", "achieved": upd["tf32"]["c_gbs"], "peak": hbm_peak, "unit": "GB/s",
                     "frac": upd["tf32"]["c_gbs"] / hbm_peak, "traffic": None,
                     "kernel": f"tc::update_kernel<tf32> (cuSsyrkLowp) m={m} k={kq}: C read+write, FP32",
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650 GB/s",
                     "tensor_tflops": upd["tf32"]["tflops"], "tensor_frac_of_tf32": upd["tf32"]["tensor_frac"],
                     "tf32_peak_tflops": tf32_peak, "bf16": upd["bf16"], "bf16_peak_tflops": bf16_peak},
    }


def batched_inputs(torch, dev, mine, sizes_all, tdt):
    """The squared-exponential kernel matrices of the batch entries `mine`, packed
    column-major into one device buffer: (buffer, sizes, offsets)."""
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
        K = torch.exp(-torch.cdist(x, x).pow(2) / (2 * 0.3 ** 2)) + 1e-4 * torch.eye(n, dtype=torch.float64,
                                                                                      device=dev)
        buf0[o:o + n * n] = K.to(tdt).reshape(-1)     # symmetric: row- and column-major agree
    return buf0, sizes, off


def batched_result(torch, cc, p, warmup, steps, peak, rank=0, world=1, pg=None, dev=None, batch=10000, nb=0):
    """10,000 squared-exponential kernel matrices K_ij = exp(-|x_i - x_j|^2 / (2 * 0.3^2))
    + 1e-4 delta_ij on n_i ~ U{8..512} points x ~ U[0,1]^3 (seed 0): factor, log det
    and inverse of every matrix in one graph launch of a batched plan, against looping
    the plain per-matrix calls (cu?potrf, cu?logdet, cu?potri) on a seeded sample of 200
    matrices, extrapolated to the whole batch by sum n^3."""
    import numpy as np
    from cucholesky import shard
    dev = dev if dev is not None else torch.device("cuda", 0)
    tdt = torch.float64 if p == "d" else torch.float32
    B = batch
    rng = np.random.default_rng(0)
    sizes_all = rng.integers(8, 513, 10000).tolist()[:B]   # the first B of the 10,000-matrix workload
    mine = shard.partition_by_cost(sizes_all, world)[rank] if world > 1 else list(range(B))
    buf0, sizes, off = batched_inputs(torch, dev, mine, sizes_all, tdt)
    buf = buf0.clone()
    h = cc.Handle()
    t0 = time.perf_counter()
    plan = cc.BatchedPlan(h, buf, sizes, off, flags=7, nb=nb)
    plan_s = time.perf_counter() - t0
    flops = float(sum(n ** 3 for n in sizes_all))    # n^3/3 (potrf) + 2n^3/3 (potri), whole batch
    for _ in range(warmup):
        buf.copy_(buf0)
        plan.run()
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        buf.copy_(buf0)
        if pg is not None:
            pg.barrier()
        ms_r, _ = timed(torch, plan.run)
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
    nb = plan.nb
    if rank != 0:
        plan.close()
        h.close()
        return None
    B_local = len(sizes)
    # accuracy on a sample: inverse residual and log det against FP64 numpy
    chk = rng.choice(B_local, min(20, B_local), replace=False)
    host = buf.cpu().numpy()
    hres = buf0.cpu().numpy()
    worst_res = worst_ld = 0.0
    eps = float(np.finfo(np.float64 if p == "d" else np.float32).eps)
    for b in chk:
        n, o = sizes[b], off[b]
        A = hres[o:o + n * n].reshape(n, n).astype(np.float64)
        X = np.tril(host[o:o + n * n].reshape(n, n, order="F").astype(np.float64))
        X = X + np.tril(X, -1).T
        kappa = np.linalg.cond(A)
        worst_res = max(worst_res, float(np.linalg.norm(np.eye(n) - A @ X) / (n * kappa * eps)))
        ref = float(np.linalg.slogdet(A)[1])
        worst_ld = max(worst_ld, float(abs(ld[b] - ref) / (n * eps * max(1.0, abs(ref)))))
    # the same work as a loop of plain per-matrix calls, on a sample
    sample = rng.choice(B_local, min(200, B_local), replace=False)
    P = p.upper()
    for b in sample[:8]:                             # untimed: first launches load their kernels
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
        ptr = buf.data_ptr() + o * buf.element_size()

        def plain():
            cc.call_potrf(h, P, "L", n, ptr, n)
            cc.call_logdet(h, P, ptr, n + 1, n)
            cc.call_potri(h, P, "L", n, ptr, n)
        loop_ms += timed(torch, plain)[0]
    frac = sum(sizes[b] ** 3 for b in sample) / flops
    loop_total_ms = loop_ms / frac
    plan.close()
    h.close()
    gfl = flops / (ms / 1e3) / 1e9
    return {
        "metric": "batched_potrf_logdet_potri_matrices_per_s", "value": B / (ms / 1e3), "unit": "matrices/s",
        "dtype": "f64" if p == "d" else "f32", "ms_per_step": ms, "steps": steps, "warmup": warmup,
        "workload": f"{B:,} squared-exponential kernel matrices, n_i ~ U{{8..512}}, lower",
        "batch": B, "sum_n3": flops, "graph_launches_per_step": 1, "nb": nb,
        "gflops": gfl,
        "loop_of_plain_calls_ms_extrapolated": loop_total_ms,
        "speedup_vs_loop": loop_total_ms / ms,
        "loop_sample": "200 matrices (seeded), cu?potrf + cu?logdet + cu?potri each, extrapolated by sum n^3",
        "failed_matrices": n_failed,
        "worst_inverse_residual_sampled": worst_res, "worst_logdet_rel_err_n_eps_sampled": worst_ld,
        "plan_build_s": plan_s,
        "roofline": {"bound": "tensor", "achieved": gfl / 1e3, "peak": peak, "unit": "TFLOP/s",
                     "frac": gfl / 1e3 / peak, "kernel": "the whole graph (potrf + logdet + potri, sum n^3 flop)",
                     "peak_source": "FP64 dense peak measured live (cuBLAS DGEMM)"},
    }


def ozaki_result(torch, cc, n, peak):
    """Large split-precision factor: dpotrf + dpotri of one FP64 SPD matrix
    A = G G^T / n + I (G uniform[-1, 1], seed 0), n = 65536 (34 GB) by default, with the
    trailing updates on the FP64 tensor cores (cuDpotrf) and as the Ozaki-sliced INT8
    emulation (cuDpotrfOzaki, its default slice count: 7 at this order); the inverse
    (cuDpotri, the same native path for both) follows the Ozaki factor.  Errors are
    estimated with 4 Gaussian probes X: the backward error ||A - L L^T||_F /
    (n eps ||A||_F) of each factor, and the inverse residual ||X - A (inv(A) X)||_F /
    (n eps ||A||_F ||inv(A) X||_F)."""
    import ctypes as C
    dev = torch.device("cuda", 0)
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

    w = make_spd_device(torch, 2048, 1, dev)      # untimed: kernel loading of both paths
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
        V = torch.empty_like(X)
        ch = 4096
        for a in range(0, n, ch):
            b = min(n, a + ch)
            V[a:b] = torch.triu(T[a:b, a:], diagonal=0) @ X[a:]
        W = torch.zeros_like(X)
        for a in range(0, n, ch):
            b = min(n, a + ch)
            W[a:] += torch.triu(T[a:b, a:], diagonal=0).T @ V[a:b]
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
            ms, (rc, info) = timed(torch, call)
            runs.append(ms)
        ms = runs[-1]
        be = factor_error(Aw)
        out[name] = {"potrf_ms": ms, "first_run_ms": runs[0], "tflops": n ** 3 / 3 / (ms / 1e3) / 1e12, "rc": rc,
                     "info": info, "backward_error_n_eps_probe": be, "bound_10": be <= 10}
    potri_ms, (rc, info) = timed(torch, lambda: cc.call_potri(h, "D", "L", n, Aw.data_ptr(), n))
    # inverse residual: Y = inv(A) X from the lower triangle of Aw (symmetric), R = X - A Y
    ch = 4096
    Y = torch.zeros_like(X)
    for a in range(0, n, ch):
        b = min(n, a + ch)
        Y[a:b] += torch.triu(Aw[a:b, a:], diagonal=0) @ X[a:]
        Y[a:] += torch.triu(Aw[a:b, a:], diagonal=1).T @ X[a:b]
    R = X - A0 @ Y
    inv_res = float(torch.linalg.norm(R).item() / (anorm * torch.linalg.norm(Y).item() * n * eps))
    h.close()
    del A0, Aw, X, Y, R
    torch.cuda.empty_cache()
    oz = out["ozaki_int8"]["tflops"]
    return {
        "metric": "ozaki_sliced_dpotrf_speedup_vs_native_dmma",
        "value": out["native_dmma"]["potrf_ms"] / out["ozaki_int8"]["potrf_ms"], "unit": "x",
        "workload": f"dpotrf + dpotri L FP64 n={n}, A=G*G^T/n+I, G~U[-1,1]", "n": n, "slices": slices,
        "arms": out, "potri_ms_after_ozaki": potri_ms, "potri_tflops": 2 * n ** 3 / 3 / (potri_ms / 1e3) / 1e12,
        "potri_rc_info": [rc, info], "inverse_residual_probe_n_eps": inv_res,
        "error_note": "4 Gaussian probes: ||A X - L L^T X||_F / (2 n eps ||A||_F); ||X - A inv(A) X||_F / "
                      "(n eps ||A||_F ||inv(A) X||_F)",
        "roofline": {"bound": "tensor", "achieved": oz, "peak": peak, "unit": "TFLOP/s (FP64-equivalent)",
                     "frac": oz / peak, "kernel": "the whole Ozaki factor (INT8 tcgen05 trailing updates)",
                     "peak_source": "FP64 dense peak measured live (cuBLAS DGEMM): above 1 means beyond "
                                    "the native FP64 roofline"},
    }


# ---------------------------------------------------------------------------------
# single-kernel modes (profiling)
# ---------------------------------------------------------------------------------
def run_syrk_only(m: int, k: int, prefix: str = "D") -> None:
    import torch
    import cucholesky as cc
    dt = torch.float64 if prefix == "D" else torch.complex128
    bh = cc.BlasHandle()
    P = torch.randn(k, m, dtype=dt, device="cuda")     # column-major m x k
    C = torch.zeros(m, m, dtype=dt, device="cuda")
    st = torch.cuda.current_stream()
    mult = 4 if prefix == "Z" else 1
    for _ in range(2):
        ms, rc = timed(torch, lambda: cc.call_rankk(bh, prefix, "L", "N", m, k, -1.0, P.data_ptr(), m, 1.0,
                                                     C.data_ptr(), m, st.cuda_stream), st)
        print(json.dumps({"kernel": "cuDsyrk L,N" if prefix == "D" else "cuZherk L,N", "m": m, "k": k, "rc": rc,
                          "ms": ms, "tflops": mult * float(m) * (m + 1) * k / (ms / 1e3) / 1e12}), flush=True)
    bh.close()


def run_single(prefix: str, n: int, uplo: str) -> None:
    import torch
    import cucholesky as cc
    from cucholesky import matgen
    p = prefix.lower()
    h = cc.Handle()
    A0 = matgen.spd_device(p, n, seed=1).to(matgen.torch_dtype(p))
    A = torch.empty_like(A0)
    for it in range(2):
        A.copy_(A0)
        ms, (rc, info) = timed(torch, lambda: cc.call_potrf(h, prefix.upper(), uplo, n, A.data_ptr(), n))
        if rc != 0 or info != 0:
            raise RuntimeError(f"cu{prefix}potrf rc={rc} info={info}")
    mult = 4 if p in "cz" else 1
    print(json.dumps({"routine": f"cu{prefix.upper()}potrf", "uplo": uplo, "n": n, "ms": ms,
                      "tflops": mult * n ** 3 / 3 / (ms / 1e3) / 1e12}), flush=True)
    h.close()


def run_syrk_lowp_only(m: int, k: int, prec: str) -> None:
    import torch
    import cucholesky as cc
    h = cc.Handle()
    p = cc.MIXED_BF16 if prec == "bf16" else cc.MIXED_TF32
    Q = (torch.rand((m, k), device="cuda", dtype=torch.float32) * 2 - 1).to(
        torch.bfloat16 if prec == "bf16" else torch.float32)
    C = torch.zeros((m, m), device="cuda", dtype=torch.float32)
    for _ in range(2):
        ms, rc = timed(torch, lambda: cc.call_syrk_lowp(h, p, m, k, -1.0, Q.data_ptr(), k, C.data_ptr(), m))
        print(json.dumps({"kernel": f"cuSsyrkLowp {prec}", "m": m, "k": k, "rc": rc, "ms": ms,
                          "tflops": float(m) * (m + 1) * k / (ms / 1e3) / 1e12,
                          "c_gbs": float(m) * (m + 1) / 2 * 8 / (ms / 1e3) / 1e9}), flush=True)
    h.close()


# ---------------------------------------------------------------------------------
# the default line
# ---------------------------------------------------------------------------------
def run_headline(args, rank, world, local):
    import ctypes as C
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
    peak, peak_clocks = fp64_peak_tflops(torch, dev, local)

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

    # the dominant kernel alone: the trailing update (tensor-core SYRK) at the shape of
    # the factorization's first outer step, k = the tuned outer block, m = n - k rows
    kk = tuned_outer_block(cc, h, "D", n)
    mk = n - kk
    syrk_ms, syrk_tflops, syrk_flops = syrk_roofline(torch, cc, "D", mk, kk, peak)
    # DRAM bytes per lower-triangle element of C measured by ncu on this kernel at
    # m = 8192 (C read + write): 15.28 at k = 512 (14.6 at k = 256 with 128 x 64
    # tiles); the panel is read once
    syrk_traffic = (15.28 if kk >= 512 else 14.6) * (float(mk) * (mk + 1) / 2) + 8.0 * mk * kk
    total_ms = t0.elapsed_time(t1)
    potrf_ms = [a.elapsed_time(b) for a, b in evs]
    if pg:
        t = torch.tensor([total_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * flops * args.steps / (total_ms / 1e3) / 1e12
    achieved = flops / (statistics.mean(potrf_ms) / 1e3) / 1e12

    # accuracy of the last factor: probe estimate of ||A - L L^T||_F / (n eps ||A||_F)
    from cucholesky import matgen
    L = matgen.factor_of(A, args.uplo)
    berr = matgen.probe_backward_error(A0, L, "d")
    del L
    torch.cuda.empty_cache()

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
            l0_, i0, o0 = hh.stats()
            t_a = time.perf_counter()
            rc, info = cc.call_host(hh, "D", "potrf", args.uplo, n, hostA.data_ptr(), n)
            t_b = time.perf_counter()
            l1_, i1, o1 = hh.stats()
            if rc != 0 or info != 0:
                raise RuntimeError(f"cuMultiGPUDpotrf rc={rc} info={info}")
            if it:
                times.append((t_b - t_a) * 1e3)
                bytes_in.append(i1 - i0)
                bytes_out.append(o1 - o0)
                nl.append(l1_ - l0_)
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

    # the reference's CPU path on this arm's own matrix, at the same order
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        import numpy as np
        Ah = np.asfortranarray(A0.cpu().numpy().T)
        times, cores, kind = cpu_reference_times(Ah, n, 3)
        del Ah
        tim = times[1:]
        cpu = {"value": n ** 3 / 3 / statistics.mean(tim) / 1e12, "unit": "TFLOP/s", "cores": cores, "kind": kind,
               "sample": f"dpotrf lower n={n} on the GPU arm's matrix (seed 0): the whole workload, "
                         f"1 untimed + {len(tim)} timed runs, {cores} threads",
               "seconds": times}
    del A, A0
    torch.cuda.empty_cache()

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        want = set(x.strip() for x in args.extras.split(",") if x.strip())
        if "potrf_n32768" in want:
            extras["potrf_n32768"] = guarded("potrf_n32768", lambda: extra_potrf_large(torch, cc, h, peak))
        if "types" in want:
            extras["types"] = guarded("types", lambda: extra_types(torch, cc, h, peak))
        if "mixed" in want:
            extras["mixed"] = guarded("mixed", lambda: mixed_result(torch, cc, h, 32768, [0.0, 1.0, 2.0, 3.0], 1, 2))
        if "batched" in want:
            extras["batched"] = {p: guarded(f"batched {p}", lambda p=p: batched_result(torch, cc, p, 2, 3, peak))
                                 for p in ("d", "s")}
        if "ozaki" in want:
            extras["ozaki"] = guarded("ozaki", lambda: ozaki_result(torch, cc, 65536, peak))

    if rank == 0:
        cfg = headline_config(n, args.uplo, world)
        cfg["outer_block"] = kk
        line = {
            "metric": "dpotrf_tflops", "value": value, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg,
            "potrf_ms": statistics.mean(potrf_ms),
            "backward_error_n_eps_probe": berr,
            "roofline": {"bound": "tensor", "achieved": syrk_tflops, "peak": peak, "unit": "TFLOP/s",
                         "frac": syrk_tflops / peak, "traffic": syrk_traffic,
                         "kernel": f"dmma::gemm_kernel<0,0,0,2> (64 x 64 tiles): trailing-update SYRK (cuDsyrk L,N) m={mk} k={kk}",
                         "kernel_ms": syrk_ms, "algorithmic_flop": syrk_flops,
                         "algorithmic_bytes": 16.0 * (float(mk) * (mk + 1) / 2) + 8.0 * mk * kk,
                         "peak_source": "FP64 dense peak measured live: best cuBLAS DGEMM 8192^3 on this GPU",
                         "peak_probe_clocks": peak_clocks},
            "potrf_fraction_of_peak": achieved / peak,
            "potrf_achieved_tflops": achieved,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": nlaunch,
            "clocks": clk.summary(),
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    h.close()
    if pg:
        pg.destroy_process_group()


def main():
    args = parse()
    if args.n is None and args.workload in ("potrf", "batched"):
        args.n = N_DEFAULT
    rank, world, local = dist_env()
    if args.syrk:
        run_syrk_only(args.syrk[0], args.syrk[1], args.syrk_type)
        return
    if args.syrk_lowp:
        run_syrk_lowp_only(int(args.syrk_lowp[0]), int(args.syrk_lowp[1]), args.syrk_lowp[2])
        return
    if args.single:
        run_single(args.single[0], int(args.single[1]), args.uplo)
        return
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.workload in ("mixed", "ozaki"):
        if rank != 0:
            return
        import torch
        import cucholesky as cc
        peak, _ = fp64_peak_tflops(torch, torch.device("cuda", 0), 0)
        if args.workload == "mixed":
            h = cc.Handle()
            r = mixed_result(torch, cc, h, args.n or 32768, [float(k) for k in args.kappa.split(",")],
                             args.warmup, args.steps)
            h.close()
        else:
            r = ozaki_result(torch, cc, args.n or 65536, peak)
        r.update({"n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                  "data": "synthetic"})
        print(json.dumps(r), flush=True)
        return
    if args.workload == "batched":
        import torch
        import cucholesky as cc
        dev = torch.device("cuda", local)
        torch.cuda.set_device(dev)
        pg = None
        if world > 1:
            # the batch shards by matrix (cost-balanced), no exchange in the data path
            import torch.distributed as dist
            from datetime import timedelta
            dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
            pg = dist
        peak, _ = fp64_peak_tflops(torch, dev, local)
        r = batched_result(torch, cc, args.dtype, args.warmup, args.steps, peak, rank, world, pg, dev,
                           batch=args.batch, nb=args.batched_nb)
        if r is not None:
            r.update({"n_gpus": world, "higher_is_better": True, "scaling": "strong" if world > 1 else "weak",
                      "vs_baseline": None, "data": "synthetic",
                      "parallelism": f"sharded by cost over {world} GPUs" if world > 1 else "single"})
            print(json.dumps(r), flush=True)
        if pg is not None:
            pg.destroy_process_group()
        return
    run_headline(args, rank, world, local)


if __name__ == "__main__":
    main()
