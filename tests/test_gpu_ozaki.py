"""cuDpotrfOzaki (FP64 Cholesky with Ozaki-sliced INT8 tensor-core trailing updates)
through the C ABI: with 8 slices the factor meets the contract's FP64 bound (backward
error <= 10 in units of n*eps) like cuDpotrf, both storages, ragged n; the info of a
non-SPD input is the oracle's; fewer slices give a factor of lower accuracy.

The tuned outer block (1024 columns at these orders) would leave a small matrix with no
trailing update at all, so the tests force 256-column outer blocks on the handle
(cuLAPACKSetPotrfBlocks), and one test runs every width the table may choose."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O
import cucholesky as cc
from cucholesky import matgen

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps


@pytest.fixture(autouse=True)
def _narrow_outer_blocks(handle):
    L = cc.lib()
    L.cuLAPACKSetPotrfBlocks.argtypes = [C.c_void_p, C.c_int]
    assert L.cuLAPACKSetPotrfBlocks(handle.value, 2) == 0
    yield
    assert L.cuLAPACKSetPotrfBlocks(handle.value, 0) == 0


def _ozaki(handle, uplo, A, slices=8):
    import torch
    L = cc.lib()
    L.cuDpotrfOzaki.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_uint64, C.c_size_t, C.c_int,
                                C.POINTER(C.c_long)]
    L.cuDpotrfOzaki.restype = C.c_int
    T = cc.to_device_colmajor(A)
    info = C.c_long(0)
    rc = L.cuDpotrfOzaki(handle.value, ord(uplo), A.shape[1], T.data_ptr(), A.shape[0], slices, C.byref(info))
    torch.cuda.synchronize()
    assert rc == 0
    return cc.to_host_colmajor(T), info.value


def _berr(A, F, uplo):
    n = A.shape[1]
    if uplo == "L":
        L = np.tril(F[:n, :n])
        R = A[:n, :n] - L @ L.T
    else:
        U = np.triu(F[:n, :n])
        R = A[:n, :n] - U.T @ U
    return np.linalg.norm(R) / (n * EPS * np.linalg.norm(A[:n, :n]))


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("n", [1, 100, 256, 257, 700, 1500, 2048])
def test_ozaki_factor_fp64_accuracy(handle, uplo, n):
    A = matgen.spd("d", n, seed=n + 11, lda=n + 3)
    F, info = _ozaki(handle, uplo, A)
    assert info == 0
    assert _berr(A, F, uplo) <= 10
    # the other triangle and the padding rows are untouched
    other = np.triu(np.ones((n, n), bool), 1) if uplo == "L" else np.tril(np.ones((n, n), bool), -1)
    assert np.array_equal(F[:n, :n][other], A[:n, :n][other])
    assert np.array_equal(F[n:], A[n:])


def test_ozaki_matches_native(handle):
    n = 1537
    A = matgen.spd("d", n, seed=5)
    F, info = _ozaki(handle, "L", A)
    T = cc.to_device_colmajor(A)
    rc, info2 = cc.call_potrf(handle, "D", "L", n, T.data_ptr(), n)
    G = cc.to_host_colmajor(T)
    assert info == info2 == 0
    d = np.abs(np.tril(F) - np.tril(G)).max() / np.abs(np.tril(G)).max()
    assert d <= 1e-12, d


def test_ozaki_not_spd_info(handle):
    n = 900
    A = matgen.spd("d", n, seed=3)
    A[700, 700] = -1.0
    ref = O.potrf("d", "L", A.copy(order="F"))
    _, info = _ozaki(handle, "L", A)
    assert info == ref == 701


def test_ozaki_fewer_slices(handle):
    n = 1024
    A = matgen.spd("d", n, seed=9)
    F8, _ = _ozaki(handle, "L", A, 8)
    F4, info = _ozaki(handle, "L", A, 4)
    assert info == 0
    b8, b4 = _berr(A, F8, "L"), _berr(A, F4, "L")
    assert b8 <= 10 < b4 < 1e10          # 4 slices: ~28-bit products, still a factor


def test_ozaki_seven_slices(handle):
    """7 slices (the default from n = 8192 on) still meet the FP64 bound at n = 4096."""
    n = 4096
    A = matgen.spd("d", n, seed=21)
    F7, info = _ozaki(handle, "L", A, 7)
    assert info == 0
    assert _berr(A, F7, "L") <= 10


@pytest.mark.parametrize("uplo", ["L", "U"])
def test_ozaki_outer_block_widths(handle, uplo):
    """Outer blocks of 256 .. 2048 columns (update launches with k up to 2048, run as
    256-wide pieces into the same accumulators) all give an FP64-accurate factor, and
    with 4 slices a visibly less accurate one (the INT8 path did the updates)."""
    L = cc.lib()
    n = 4500
    A = matgen.spd("d", n, seed=21, lda=n + 1)
    for sub in (2, 4, 8, 16):
        assert L.cuLAPACKSetPotrfBlocks(handle.value, sub) == 0
        F, info = _ozaki(handle, uplo, A, 7)
        assert info == 0
        assert _berr(A, F, uplo) <= 10, sub
        F4, info = _ozaki(handle, uplo, A, 4)
        assert info == 0 and 10 < _berr(A, F4, uplo) < 1e10, sub

