"""cu?trsm and cu?trmm2 (include/blas.h, reference blas/dtrsm.c:218 and
blas/dtrmm.c:374) through the C ABI, for every side, uplo, op and diag, s/d/c/z,
against numpy.  The unreferenced triangle of A (and its diagonal when diag = U) holds
NaN, so a read of it would show."""
from __future__ import annotations

import itertools

import numpy as np
import pytest

import cucholesky as cc

pytestmark = pytest.mark.gpu

DT = {"S": np.float32, "D": np.float64, "C": np.complex64, "Z": np.complex128}


@pytest.fixture(scope="module")
def bh():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    h = cc.BlasHandle()
    yield h
    h.close()


def _tri(p, k, uplo, diag, rng):
    dt = DT[p]
    M = rng.uniform(-1, 1, (k, k))
    if p in "CZ":
        M = M + 1j * rng.uniform(-1, 1, (k, k))
    M = M / np.sqrt(k)
    M[np.diag_indices(k)] = 2.0 + rng.uniform(0, 1, k)       # well conditioned
    T = np.tril(M) if uplo == "L" else np.triu(M)
    stored = T.copy()
    other = np.triu(np.ones((k, k), bool), 1) if uplo == "L" else np.tril(np.ones((k, k), bool), -1)
    stored[other] = np.nan
    if diag == "U":
        T[np.diag_indices(k)] = 1.0
        stored[np.diag_indices(k)] = np.nan
    return T.astype(dt), np.asfortranarray(stored.astype(dt))


def _op(T, trans):
    return T if trans == "N" else (T.T if trans == "T" else T.conj().T)


COMBOS = list(itertools.product("SDCZ", "LR", "LU", "NTC", "NU"))


@pytest.mark.parametrize("p,side,uplo,trans,diag", COMBOS)
def test_trsm(bh, p, side, uplo, trans, diag):
    import torch
    rng = np.random.default_rng(hash((p, side, uplo, trans, diag)) % 2**32)
    m, n = 203, 71
    k = m if side == "L" else n
    T, stored = _tri(p, k, uplo, diag, rng)
    B = rng.uniform(-1, 1, (m, n)).astype(DT[p])
    if p in "CZ":
        B = (B + 1j * rng.uniform(-1, 1, (m, n))).astype(DT[p])
    alpha = 0.75 if p in "SD" else 0.75 - 0.25j
    TA = cc.to_device_colmajor(stored)
    TB = cc.to_device_colmajor(np.asfortranarray(B))
    rc = cc.call_trsm(bh, p, side, uplo, trans, diag, m, n, alpha, TA.data_ptr(), k, TB.data_ptr(), m)
    torch.cuda.synchronize()
    assert rc == 0
    X = cc.to_host_colmajor(TB).astype(np.complex128 if p in "CZ" else np.float64)
    opT = _op(T.astype(np.complex128 if p in "CZ" else np.float64), trans)
    ref = alpha * (np.linalg.solve(opT, B) if side == "L" else np.linalg.solve(opT.T, B.T).T)
    eps = np.finfo(DT[p]).eps
    assert np.isfinite(X).all()
    assert np.abs(X - ref).max() <= 50 * max(m, n) * eps * np.abs(ref).max()


@pytest.mark.parametrize("p,side,uplo,trans,diag", COMBOS)
def test_trmm2(bh, p, side, uplo, trans, diag):
    import torch
    rng = np.random.default_rng(hash((p, side, uplo, trans, diag, 1)) % 2**32)
    m, n = 150, 67
    k = m if side == "L" else n
    T, stored = _tri(p, k, uplo, diag, rng)
    B = rng.uniform(-1, 1, (m, n)).astype(DT[p])
    alpha = 1.5 if p in "SD" else 1.5 + 0.5j
    TA = cc.to_device_colmajor(stored)
    TB = cc.to_device_colmajor(np.asfortranarray(B))
    TX = cc.to_device_colmajor(np.asfortranarray(np.full((m, n), 7.0, dtype=DT[p])))
    rc = cc.call_trmm2(bh, p, side, uplo, trans, diag, m, n, alpha, TA.data_ptr(), k, TB.data_ptr(), m,
                       TX.data_ptr(), m)
    torch.cuda.synchronize()
    assert rc == 0
    X = cc.to_host_colmajor(TX).astype(np.complex128 if p in "CZ" else np.float64)
    opT = _op(T.astype(np.complex128 if p in "CZ" else np.float64), trans)
    Bd = B.astype(X.dtype)
    ref = alpha * (opT @ Bd if side == "L" else Bd @ opT)
    eps = np.finfo(DT[p]).eps
    bound = 4 * k * eps * (np.abs(alpha) * (np.abs(opT) @ np.abs(Bd) if side == "L" else np.abs(Bd) @ np.abs(opT)))
    assert (np.abs(X - ref) <= bound + 1e-30).all()


def test_trsm_argument_errors(bh):
    import ctypes as C
    calls = []
    XERBLA = C.CFUNCTYPE(None, C.c_char_p, C.c_long)
    cb = XERBLA(lambda name, info: calls.append((name.decode(), info)))
    lib = cc.lib()
    xer = C.c_void_p.in_dll(lib, "xerbla")
    old = xer.value
    xer.value = C.cast(cb, C.c_void_p).value
    try:
        assert cc.call_trsm(bh, "D", "L", "L", "N", "N", 10, 5, 1.0, 0, 9, 0, 10) == cc.CUDA_ERROR_INVALID_VALUE
        assert calls[-1] == ("cuDtrsm", 9)
        assert cc.call_trsm(bh, "D", "R", "L", "N", "N", 10, 5, 1.0, 0, 5, 0, 9) == cc.CUDA_ERROR_INVALID_VALUE
        assert calls[-1] == ("cuDtrsm", 11)
        assert cc.call_trmm2(bh, "D", "L", "L", "N", "N", 10, 5, 1.0, 0, 10, 0, 10, 0, 9) == \
            cc.CUDA_ERROR_INVALID_VALUE
        assert calls[-1] == ("cuDtrmm2", 13)
    finally:
        xer.value = old
