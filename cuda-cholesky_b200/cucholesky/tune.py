"""Tuner for libcucholesky.so's tuning table (the counterpart of the reference's
blas/config.c, which timed its kernels at build time and wrote include/config.h).

For each type and order it times ?potrf (CUDA events around cu?potrf, best of a few
runs after a warm-up) with every candidate outer-block size (cuLAPACKSetPotrfBlocks),
keeps the fastest, and writes the table in the library's text format:

    cucholesky-tuning 1
    potrf D 0 2
    potrf D 6144 3
    ...

one row per measured order, with n_min at the geometric midpoint between neighbouring
orders.  Load the file with cuLAPACKLoadTuning or the CUCHOLESKY_TUNING environment
variable.  Inputs: cu?latmc (condition number 100) on the device.

    PYTHONPATH=cuda-cholesky_b200 python -m cucholesky.tune --types D \
        --sizes 4096,8192,16384,32768 --out b200.tuning
"""
from __future__ import annotations

import argparse
import ctypes as C
import math

import cucholesky as cc

CANDIDATES = (2, 3, 4, 6, 8)
_DT = {"S": "float32", "D": "float64", "C": "complex64", "Z": "complex128"}


def _declare(L):
    L.cuLAPACKSetPotrfBlocks.argtypes = [C.c_void_p, C.c_int]
    L.cuLAPACKSetPotrfBlocks.restype = C.c_int
    L.cuLAPACKGetPotrfBlocks.argtypes = [C.c_void_p, C.c_char, C.c_size_t, C.POINTER(C.c_int)]
    L.cuLAPACKGetPotrfBlocks.restype = C.c_int
    L.cuLAPACKLoadTuning.argtypes = [C.c_char_p]
    L.cuLAPACKLoadTuning.restype = C.c_int


def time_potrf(h, prefix: str, n: int, sub: int, reps: int = 3) -> float:
    """Best event-timed ms of cu<prefix>potrf (lower) of one cu?latmc matrix."""
    import torch
    L = cc.lib()
    _declare(L)
    assert L.cuLAPACKSetPotrfBlocks(h.value, sub) == 0
    dt = getattr(torch, _DT[prefix])
    A0 = torch.empty((n, n), dtype=dt, device="cuda")
    g = cc.Rng(32 if prefix in "SC" else 64, seed=n)
    assert cc.call_latmc(prefix, g, n, 100.0, A0.data_ptr(), n) == 0
    g.close()
    A = torch.empty_like(A0)
    best = math.inf
    for it in range(reps + 1):
        A.copy_(A0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rc, info = cc.call_potrf(h, prefix, "L", n, A.data_ptr(), n)
        e1.record()
        torch.cuda.synchronize()
        if rc != 0 or info != 0:
            raise RuntimeError(f"cu{prefix}potrf n={n} sub={sub}: rc={rc} info={info}")
        if it:
            best = min(best, e0.elapsed_time(e1))
    assert L.cuLAPACKSetPotrfBlocks(h.value, 0) == 0
    return best


def table_rows(prefix: str, results: dict[int, int]) -> list[str]:
    """Rows for one type from {n: best sub}: n_min at geometric midpoints."""
    ns = sorted(results)
    rows = []
    for i, n in enumerate(ns):
        n_min = 0 if i == 0 else int(round(math.sqrt(ns[i - 1] * n)))
        rows.append(f"potrf {prefix} {n_min} {results[n]}")
    return rows


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--types", default="D")
    ap.add_argument("--sizes", default="4096,8192,16384,32768")
    ap.add_argument("--candidates", default=",".join(str(c) for c in CANDIDATES))
    ap.add_argument("--out", required=True)
    args = ap.parse_args(argv)
    import torch
    torch.cuda.init()
    h = cc.Handle()
    sizes = [int(x) for x in args.sizes.split(",")]
    cands = [int(x) for x in args.candidates.split(",")]
    lines = ["cucholesky-tuning 1", f"# {torch.cuda.get_device_name(0)}; ?potrf outer block in diagonal blocks"]
    for prefix in args.types.upper():
        best = {}
        for n in sizes:
            times = {s: time_potrf(h, prefix, n, s) for s in cands}
            best[n] = min(times, key=times.get)
            print(f"{prefix} n={n}: " + ", ".join(f"{s}: {t:.2f} ms" for s, t in times.items()), flush=True)
        lines += table_rows(prefix, best)
    with open(args.out, "w") as f:
        f.write("\n".join(lines) + "\n")
    h.close()


if __name__ == "__main__":
    main()
