"""Generate the golden vectors in tests/golden/ from the reference's own CPU
library (oracle/_ref/libref.so, compiled from the reference's lapack/*.c and
blas/*.c by oracle/ref.mk).

    python tests/golden/make_golden.py

The reference ships no golden vector files (its tests build matrices with
glibc rand(), test/lapack/util/dlatmc.c); these fixtures freeze its outputs on
small seeded inputs so that parity can be checked where the reference tree is
not available.  Each case stores the input, the reference's potrf factor and
info, its potri result and info, and its logdet of the factor.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "cuda-cholesky_b200"))

import oracle as O  # noqa: E402
from cucholesky import matgen  # noqa: E402

SIZES = [1, 2, 7, 31, 32, 33, 64, 65]


def cases():
    for p in "sdcz":
        for u in "LU":
            for n in SIZES:
                yield p, u, n, n, None
            yield p, u, 45, 50, None          # lda > n
            yield p, u, 70, 70, 40            # not positive definite at row/col 40
    for u in "LU":
        yield "d", u, 150, 150, None          # crosses the GPU path's block boundary


def main() -> None:
    if not O.available("reference"):
        raise SystemExit("oracle/_ref/libref.so is not built (make -f oracle/Makefile ref REF=<reference tree>)")
    out = {}
    for p, u, n, lda, bad in cases():
        A = matgen.spd(p, n, seed=1000 + n, lda=lda)
        if bad is not None:
            A[bad, bad] = -1.0
        F = A.copy(order="F")
        info = O.potrf(p, u, F, lda=lda, impl="reference")
        key = f"{p}{u}_{n}_{lda}" + (f"_bad{bad}" if bad is not None else "")
        out[key + "_A"] = A
        out[key + "_F"] = F
        out[key + "_info"] = np.array(info)
        if info == 0:
            X = F.copy(order="F")
            out[key + "_Xinfo"] = np.array(O.potri(p, u, X, impl="reference"))
            out[key + "_X"] = X
            out[key + "_logdet"] = np.array(O.logdet(p, F.ravel(order="F"), lda + 1, n, impl="reference"))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_small.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays")


if __name__ == "__main__":
    main()
