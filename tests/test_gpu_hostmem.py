"""Host-memory routines cuMultiGPU?potrf / ?trtri / ?lauum / ?potri (reference
include/lapack.h:117-158; tests modelled on test/lapack/cumultigpu?potrf.c:40-90):
the matrix lives in host memory, the result must equal the oracle within the
contract's bounds and, while the factorization runs as one panel (n < 2048), equal
bit for bit the single-GPU routine on the same values; the other triangle and the
padding rows stay untouched; numerical failure returns CUDA_ERROR_INVALID_VALUE
with the oracle's info."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import cucholesky as cc
from cucholesky import matgen

pytestmark = pytest.mark.gpu

EPS = {"s": np.finfo(np.float32).eps, "d": np.finfo(np.float64).eps,
       "c": np.finfo(np.float32).eps, "z": np.finfo(np.float64).eps}


@pytest.fixture(scope="module")
def hosth():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    m = cc.MultiGPU([0])
    hh = cc.HostHandle(m)
    yield hh
    hh.close()
    m.close()


def _tri(u):
    return np.tril if u == "L" else np.triu


def _other(n, u):
    return np.triu(np.ones((n, n), bool), 1) if u == "L" else np.tril(np.ones((n, n), bool), -1)


def _device_result(handle, fn, p, u, A, *extra):
    """The single-GPU routine on the same values, with the leading dimension the
    host-memory routine stages with (n rounded up to 32)."""
    import torch
    n = A.shape[1]
    ldd = -(-n // 32) * 32
    B = np.zeros((ldd, n), dtype=A.dtype, order="F")
    B[:n, :n] = A[:n, :n]
    T = cc.to_device_colmajor(B)
    rc, info = getattr(cc, f"call_{fn}")(handle, p.upper(), u, *extra, n, T.data_ptr(), ldd)
    torch.cuda.synchronize()
    return cc.to_host_colmajor(T)[:n, :n], rc, info


@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("u", ["L", "U"])
def test_host_potrf_potri(hosth, handle, p, u):
    for n in (1, 65, 300, 777):
        lda = n + 3
        A = matgen.spd(p, n, seed=n, lda=lda)
        H = A.copy(order="F")
        rc, info = cc.call_host(hosth, p.upper(), "potrf", u, n, H.ctypes.data, lda)
        assert rc == 0 and info == 0, (n, rc, info)
        Fo = A.copy(order="F")
        assert O.potrf(p, u, Fo, lda=lda) == 0
        assert matgen.backward_error(A, H, u) <= 10, n
        d = np.abs(_tri(u)(H[:n, :n] - Fo[:n, :n])).max()
        assert d <= 50 * n * EPS[p] * np.abs(A[:n, :n]).max(), (n, d)
        # untouched: the other triangle and the padding rows
        assert np.array_equal(H[:n, :n][_other(n, u)], A[:n, :n][_other(n, u)]), n
        assert np.array_equal(H[n:, :], A[n:, :]), n
        # same kernels, same values: bit-identical to the single-GPU routine
        Fd, rc2, info2 = _device_result(handle, "potrf", p, u, A)
        assert rc2 == 0 and info2 == 0
        assert np.array_equal(_tri(u)(H[:n, :n]), _tri(u)(Fd)), n
        # inverse in host memory
        X = H.copy(order="F")
        rc, info = cc.call_host(hosth, p.upper(), "potri", u, n, X.ctypes.data, lda)
        assert rc == 0 and info == 0
        assert matgen.inverse_residual(A, X, u) <= 10, n
        assert np.array_equal(X[:n, :n][_other(n, u)], A[:n, :n][_other(n, u)]), n
        assert np.array_equal(X[n:, :], A[n:, :]), n


@pytest.mark.parametrize("p", list("dz"))
@pytest.mark.parametrize("u", ["L", "U"])
def test_host_trtri_lauum(hosth, handle, p, u):
    for n, diag in ((129, "N"), (300, "U"), (515, "N")):
        lda = n + 1
        A = matgen.spd(p, n, seed=n, lda=lda)
        F = A.copy(order="F")
        assert O.potrf(p, u, F, lda=lda) == 0
        T = F.copy(order="F")
        rc, info = cc.call_host(hosth, p.upper(), "trtri", u, n, T.ctypes.data, lda, diag)
        assert rc == 0 and info == 0
        To = F.copy(order="F")
        assert O.trtri(p, u, To, diag) == 0
        d = np.abs(_tri(u)(T[:n, :n] - To[:n, :n])).max() / np.abs(To[:n, :n]).max()
        assert d <= 1e3 * n * EPS[p], (n, d)
        Td, rc2, _ = _device_result(handle, "trtri", p, u, F, diag)
        assert rc2 == 0 and np.array_equal(_tri(u)(T[:n, :n]), _tri(u)(Td))
        Lm = F.copy(order="F")
        rc, info = cc.call_host(hosth, p.upper(), "lauum", u, n, Lm.ctypes.data, lda)
        assert rc == 0 and info == 0
        Lo = F.copy(order="F")
        O.lauum(p, u, Lo)
        d = np.abs(_tri(u)(Lm[:n, :n] - Lo[:n, :n])).max() / np.abs(Lo[:n, :n]).max()
        assert d <= 100 * n * EPS[p], (n, d)
        assert np.array_equal(Lm[n:, :], F[n:, :])


@pytest.mark.parametrize("u", ["L", "U"])
def test_host_pinned_overlapped_copy_back(hosth, handle, u):
    """Page-locked host memory takes the overlapped path (each block column of the
    factor copied back behind the work that finishes it): same bits as the
    single-GPU routine, and the bytes moved are the triangle's trapezoids."""
    import torch
    n, lda = 1500, 1502
    A = matgen.spd("d", n, seed=7, lda=lda)
    P = torch.empty((n, lda), dtype=torch.float64, pin_memory=True)   # column-major (lda, n)
    P.copy_(torch.from_numpy(np.ascontiguousarray(A.T)))
    _, h2d0, d2h0 = hosth.stats()
    rc, info = cc.call_host(hosth, "D", "potrf", u, n, P.data_ptr(), lda)
    assert rc == 0 and info == 0
    _, h2d1, d2h1 = hosth.stats()
    H = np.asfortranarray(P.numpy().T)
    assert matgen.backward_error(A, H, u) <= 10
    Fd, _, _ = _device_result(handle, "potrf", "d", u, A)
    assert np.array_equal(_tri(u)(H[:n, :n]), _tri(u)(Fd))
    assert np.array_equal(H[:n, :n][_other(n, u)], A[:n, :n][_other(n, u)])
    assert np.array_equal(H[n:, :], A[n:, :])
    tri = 8 * n * (n + 1) // 2
    assert tri <= h2d1 - h2d0 <= tri + 8 * n * 256          # 256-column trapezoids
    assert tri <= d2h1 - d2h0 <= tri + 8 * n * 128          # 128-column diagonal blocks


@pytest.mark.parametrize("p", list("dc"))
@pytest.mark.parametrize("u", ["L", "U"])
def test_host_not_positive_definite(hosth, p, u):
    n, lda = 400, 401
    A = matgen.spd(p, n, seed=3, lda=lda)
    A[250, 250] = -1.0
    H = A.copy(order="F")
    rc, info = cc.call_host(hosth, p.upper(), "potrf", u, n, H.ctypes.data, lda)
    Fo = A.copy(order="F")
    want = O.potrf(p, u, Fo, lda=lda)
    assert want > 0
    assert rc == cc.CUDA_ERROR_INVALID_VALUE and info == want
    k = info - 1
    d = np.abs(_tri(u)(H[:k, :k] - Fo[:k, :k])).max()
    assert d <= 50 * n * EPS[p] * np.abs(A[:n, :n]).max()


@pytest.mark.parametrize("u", ["L", "U"])
def test_host_singular_trtri_and_potri_leave_a(hosth, u):
    n, lda = 300, 300
    A = matgen.spd("d", n, seed=5, lda=lda)
    F = A.copy(order="F")
    assert O.potrf("d", u, F, lda=lda) == 0
    F[123, 123] = 0.0
    want = O.trtri("d", u, F.copy(order="F"), "N")
    assert want > 0
    for routine in ("trtri", "potri"):
        T = F.copy(order="F")
        rc, info = cc.call_host(hosth, "D", routine, u, n, T.ctypes.data, lda)
        assert rc == cc.CUDA_ERROR_INVALID_VALUE and info == want, routine
        assert np.array_equal(T, F), routine


def test_device_list_and_sync(hosth):
    m = cc.MultiGPU([0, 0])
    assert m.count() == 2
    assert m.synchronize() == 0
    hh = cc.HostHandle(m)
    A = matgen.spd("s", 64, seed=1)
    rc, info = cc.call_host(hh, "S", "potrf", "L", 64, A.ctypes.data, 64)
    assert rc == 0 and info == 0
    assert hh.synchronize() == 0
    hh.close()
    m.close()
    assert hosth.synchronize() == 0


def _pinned_colmajor(A):
    import torch
    lda, n = A.shape
    P = torch.empty((n, lda), dtype=getattr(torch, str(A.dtype)), pin_memory=True)
    P.copy_(torch.from_numpy(np.ascontiguousarray(A.T)))
    return P


@pytest.mark.parametrize("p", list("dz"))
@pytest.mark.parametrize("u", ["L", "U"])
def test_host_streamed_tall_panels(hosth, p, u):
    """Page-locked A with n > 2048: copied in as tall panels (1024 columns up to the
    middle column, then the rest) and factored left-looking panel by panel.  The
    factor meets the backward-error bound; the other triangle and the padding are
    untouched; a failure in a later panel reports its global position."""
    n, lda = 4500, 4502
    A = matgen.spd(p, n, seed=11, lda=lda)
    P = _pinned_colmajor(A)
    _, h2d0, d2h0 = hosth.stats()
    rc, info = cc.call_host(hosth, p.upper(), "potrf", u, n, P.data_ptr(), lda)
    assert rc == 0 and info == 0
    _, h2d1, d2h1 = hosth.stats()
    H = np.asfortranarray(P.numpy().T)
    assert matgen.backward_error(A, H, u) <= 10
    assert np.array_equal(H[:n, :n][_other(n, u)], A[:n, :n][_other(n, u)])
    assert np.array_equal(H[n:, :], A[n:, :])
    esz = A.itemsize
    tri = esz * n * (n + 1) // 2
    assert tri <= h2d1 - h2d0 <= tri + esz * n * 256
    assert tri <= d2h1 - d2h0 <= tri + esz * n * 128
    # not positive definite at 3001 (inside the last panel) and at 1500 (second panel)
    for bad in (3000, 1500):
        B = A.copy(order="F")
        B[bad, bad] = -1.0
        Q = _pinned_colmajor(B)
        rc, info = cc.call_host(hosth, p.upper(), "potrf", u, n, Q.data_ptr(), lda)
        assert rc == cc.CUDA_ERROR_INVALID_VALUE and info == bad + 1, (bad, rc, info)
