"""The BLAS layer (include/blas.h: cu?gemm2, cu?syrk, cu?herk) through the C ABI,
against numpy in FP64/complex128, with the reference tests' per-element bound
(test/blas/cudgemm.c:224-230: |D - Dref| <= (2k+2) * eps * (|alpha| |A||B| + |beta| |C|))."""
from __future__ import annotations

import numpy as np
import pytest

import cucholesky as cc
from cucholesky import matgen

pytestmark = pytest.mark.gpu

EPS = {"S": np.finfo(np.float32).eps, "D": np.finfo(np.float64).eps,
       "C": np.finfo(np.float32).eps, "Z": np.finfo(np.float64).eps}
NP = {"S": np.float32, "D": np.float64, "C": np.complex64, "Z": np.complex128}


@pytest.fixture(scope="module")
def bh():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    h = cc.BlasHandle()
    yield h
    h.close()


def _rand(p, shape, rng):
    x = rng.standard_normal(shape)
    if p in "CZ":
        x = x + 1j * rng.standard_normal(shape)
    return np.asfortranarray(x.astype(NP[p]))


def _op(X, t):
    return X if t == "N" else (X.T if t == "T" else X.conj().T)


@pytest.mark.parametrize("p", list("SDCZ"))
def test_gemm2(bh, p):
    import torch
    rng = np.random.default_rng(1)
    for (m, n, k) in ((1, 1, 1), (130, 70, 33), (257, 129, 200), (64, 64, 0)):
        for ta in "NTC":
            for tb in "NTC":
                A = _rand(p, (m, k) if ta == "N" else (k, m), rng)
                B = _rand(p, (k, n) if tb == "N" else (n, k), rng)
                Cm = _rand(p, (m, n), rng)
                alpha, beta = (0.7 - 0.2j, -1.3 + 0.5j) if p in "CZ" else (0.7, -1.3)
                tA, tB, tC = (cc.to_device_colmajor(X) for X in (A, B, Cm))
                tD = torch.zeros_like(tC)
                rc = cc.call_gemm2(bh, p, ta, tb, m, n, k, alpha, tA.data_ptr(), A.shape[0], tB.data_ptr(),
                                   B.shape[0], beta, tC.data_ptr(), m, tD.data_ptr(), m)
                assert rc == 0
                torch.cuda.synchronize()
                D = cc.to_host_colmajor(tD)
                A64, B64, C64 = (X.astype(np.complex128 if p in "CZ" else np.float64) for X in (A, B, Cm))
                ref = alpha * _op(A64, ta) @ _op(B64, tb) + beta * C64
                bound = (2 * k + 2) * EPS[p] * (abs(alpha) * np.abs(_op(A64, ta)) @ np.abs(_op(B64, tb))
                                               + abs(beta) * np.abs(C64)) + 1e-30
                assert np.all(np.abs(D - ref) <= 4 * bound), (m, n, k, ta, tb)


@pytest.mark.parametrize("p", list("SDCZ"))
def test_syrk_herk(bh, p):
    import torch
    rng = np.random.default_rng(2)
    herm = p in "CZ"
    for (n, k) in ((1, 1), (100, 17), (300, 128), (129, 257)):
        for uplo in "LU":
            for tr in ("NC" if herm else "NT"):
                A = _rand(p, (n, k) if tr == "N" else (k, n), rng)
                Cm = _rand(p, (n, n), rng)
                tA, tC = cc.to_device_colmajor(A), cc.to_device_colmajor(Cm)
                rc = cc.call_rankk(bh, p, uplo, tr, n, k, -1.0, tA.data_ptr(), A.shape[0], 0.5, tC.data_ptr(), n)
                assert rc == 0
                torch.cuda.synchronize()
                R = cc.to_host_colmajor(tC)
                A64 = A.astype(np.complex128 if herm else np.float64)
                opA = A64 if tr == "N" else (A64.conj().T if herm else A64.T)
                ref = -1.0 * opA @ (opA.conj().T if herm else opA.T) + 0.5 * Cm.astype(A64.dtype)
                if herm:   # a Hermitian result: the diagonal's imaginary part is zero
                    ref[np.diag_indices(n)] = ref[np.diag_indices(n)].real
                tri = np.tril if uplo == "L" else np.triu
                mask = tri(np.ones((n, n), bool))
                bound = (2 * k + 2) * EPS[p] * (np.abs(opA) @ np.abs(opA).T + 0.5 * np.abs(Cm)) + 1e-30
                assert np.all(np.abs(R - ref)[mask] <= 4 * bound[mask]), (n, k, uplo, tr)
                assert np.array_equal(R[~mask], Cm[~mask])      # other triangle untouched
                if herm:
                    assert np.all(np.diag(R).imag == 0)


def test_blas_argument_errors(bh):
    import ctypes as C
    assert cc.call_gemm2(bh, "D", "N", "N", 10, 10, 10, 1.0, 0, 5, 0, 10, 0.0, 0, 10, 0, 10) == 1
    assert cc.call_rankk(bh, "D", "L", "N", 10, 4, 1.0, 0, 5, 0.0, 0, 10) == 1
    assert cc.call_rankk(bh, "Z", "L", "T", 10, 4, 1.0, 0, 10, 0.0, 0, 10) == 1
