"""Parity of the GPU path (through the C ABI of libcucholesky.so) with the oracle:
golden vectors frozen from the reference library, the plain-C restatement on
seeded inputs, bit-exact info, and the error bounds of the contract
(backward error and inverse residual <= 10 in units of n*eps, logdet relative
error <= 100*n*eps)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import cucholesky as cc
from cucholesky import matgen

pytestmark = pytest.mark.gpu

EPS = {"s": np.finfo(np.float32).eps, "d": np.finfo(np.float64).eps,
       "c": np.finfo(np.float32).eps, "z": np.finfo(np.float64).eps}


def _tri(u):
    return np.tril if u == "L" else np.triu


def gpu_call(handle, fn, p, u, A, *extra):
    """Run cu<P><fn> on a copy of the column-major numpy matrix A (shape (lda, n));
    returns (result matrix, info)."""
    import torch
    T = cc.to_device_colmajor(A)
    n = A.shape[1]
    rc, info = getattr(cc, f"call_{fn}")(handle, p.upper(), u, *extra, n, T.data_ptr(), A.shape[0])
    assert rc == 0, f"cu{p.upper()}{fn} returned {rc}"
    torch.cuda.synchronize()
    return cc.to_host_colmajor(T), info


def gpu_logdet(handle, p, F):
    import torch
    T = cc.to_device_colmajor(F)
    rc, out = cc.call_logdet(handle, p.upper(), T.data_ptr(), F.shape[0] + 1, F.shape[1])
    assert rc == 0
    torch.cuda.synchronize()
    return float(out.value)


def fp64_logdet(F):
    n = F.shape[1]
    return 2.0 * float(np.sum(np.log(np.real(np.diag(F[:n, :n])).astype(np.float64))))


def _golden_keys(golden):
    return sorted({k.rsplit("_", 1)[0] for k in golden.files if k.endswith("_info")})


def test_golden_vectors(handle, golden):
    for key in _golden_keys(golden):
        p, u = key[0], key[1]
        n, lda = (int(v) for v in key.split("_")[1:3])
        A = golden[key + "_A"]
        F, info = gpu_call(handle, "potrf", p, u, A)
        assert info == int(golden[key + "_info"]), key
        Fg = golden[key + "_F"]
        if info != 0:
            k = info - 1
            d = np.abs(_tri(u)(F[:k, :k] - Fg[:k, :k])).max() if k else 0.0
            assert d <= 50 * n * EPS[p] * np.abs(A[:n, :n]).max(), (key, d)
            continue
        be = matgen.backward_error(A, F, u)
        assert be <= 10, (key, be)
        d = np.abs(_tri(u)(F[:n, :n] - Fg[:n, :n])).max()
        assert d <= 50 * n * EPS[p] * np.abs(A[:n, :n]).max(), (key, d)
        # the other triangle and the padding rows are untouched
        other = np.triu(np.ones((n, n), bool), 1) if u == "L" else np.tril(np.ones((n, n), bool), -1)
        assert np.array_equal(F[:n, :n][other], A[:n, :n][other]), key
        assert np.array_equal(F[n:, :], A[n:, :]), key
        X, xinfo = gpu_call(handle, "potri", p, u, F)
        assert xinfo == int(golden[key + "_Xinfo"]) == 0
        ir = matgen.inverse_residual(A, X, u)
        assert ir <= 10, (key, ir)
        ld = gpu_logdet(handle, p, F)
        ref = fp64_logdet(Fg)
        assert abs(ld - ref) <= 100 * n * EPS[p] * max(1.0, abs(ref)), (key, ld, ref)


SIZES = [1, 5, 63, 64, 65, 127, 128, 129, 200, 256, 257, 300, 513]


@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("u", ["L", "U"])
def test_ragged_sizes_vs_oracle(handle, p, u):
    for n in SIZES:
        lda = n + (3 if n % 2 else 0)
        A = matgen.spd(p, n, seed=n, lda=lda)
        F, info = gpu_call(handle, "potrf", p, u, A)
        Fo = A.copy(order="F")
        assert info == O.potrf(p, u, Fo, lda=lda) == 0
        be = matgen.backward_error(A, F, u)
        assert be <= 10, (n, be)
        d = np.abs(_tri(u)(F[:n, :n] - Fo[:n, :n])).max()
        assert d <= 50 * n * EPS[p] * np.abs(A[:n, :n]).max(), (n, d)
        X, xinfo = gpu_call(handle, "potri", p, u, F)
        assert xinfo == 0
        assert matgen.inverse_residual(A, X, u) <= 10, n
        Xo = Fo.copy(order="F")
        O.potri(p, u, Xo)
        d = np.abs(_tri(u)(X[:n, :n] - Xo[:n, :n])).max() / np.abs(Xo[:n, :n]).max()
        assert d <= 1e3 * n * EPS[p], (n, d)
        ld, ref = gpu_logdet(handle, p, F), fp64_logdet(Fo)
        assert abs(ld - ref) <= 100 * n * EPS[p] * max(1.0, abs(ref)), (n, ld, ref)


@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("u", ["L", "U"])
def test_info_non_spd(handle, p, u):
    n = 300
    for bad in (0, 5, 127, 128, 129, 250, 299):
        A = matgen.spd(p, n, seed=11)
        A[bad, bad] = -1.0
        F, info = gpu_call(handle, "potrf", p, u, A)
        Fo = A.copy(order="F")
        assert info == O.potrf(p, u, Fo) == bad + 1
        k = info - 1
        if k:
            d = np.abs(_tri(u)(F[:k, :k] - Fo[:k, :k])).max()
            assert d <= 50 * n * EPS[p] * np.abs(A).max()
    A = matgen.spd(p, n, seed=12)
    A[200, 200] = np.nan
    _, info = gpu_call(handle, "potrf", p, u, A)
    assert info == 201


def test_config1_fp64_n2048(handle):
    """FP64 n=2048, lower: potrf + potri + logdet against the oracle, and the
    non-SPD variant A[1000][1000] = -1 -> info 1001."""
    n = 2048
    A = matgen.spd("d", n, seed=0)
    F, info = gpu_call(handle, "potrf", "d", "L", A)
    Fo = A.copy(order="F")
    assert info == O.potrf("d", "L", Fo) == 0
    assert matgen.backward_error(A, F, "L") <= 10
    X, xinfo = gpu_call(handle, "potri", "d", "L", F)
    assert xinfo == 0
    assert matgen.inverse_residual(A, X, "L") <= 10
    ld, ref = gpu_logdet(handle, "d", F), O.logdet("d", Fo.ravel(order="F"), n + 1, n)
    assert abs(ld - ref) <= 100 * n * EPS["d"] * abs(ref)
    B = A.copy(order="F")
    B[1000, 1000] = -1.0
    for u in "LU":
        _, info = gpu_call(handle, "potrf", "d", u, B)
        assert info == 1001


@pytest.mark.parametrize("p", list("sdcz"))
def test_trtri_and_lauum(handle, p):
    for u in "LU":
        for n in (70, 300):
            A = matgen.spd(p, n, seed=21)
            Fo = A.copy(order="F")
            O.potrf(p, u, Fo)
            for diag in "NU":
                T, info = gpu_call(handle, "trtri", p, u, Fo, diag)
                To = Fo.copy(order="F")
                assert info == O.trtri(p, u, To, diag) == 0
                d = np.abs(_tri(u)(T - To)).max() / np.abs(To).max()
                assert d <= 1e3 * n * EPS[p], (u, n, diag, d)
                if diag == "U":   # the diagonal itself is not referenced or written
                    assert np.array_equal(np.diag(T), np.diag(Fo))
            Lm, _ = gpu_call(handle, "lauum", p, u, Fo)
            Lo = Fo.copy(order="F")
            O.lauum(p, u, Lo)
            d = np.abs(_tri(u)(Lm - Lo)).max() / np.abs(Lo).max()
            assert d <= 100 * n * EPS[p], (u, n, d)


def test_trtri_singular_info(handle):
    n = 300
    T = np.asfortranarray(np.tril(matgen.spd("d", n, seed=6)))
    T[10, 10] = 0.0
    T[270, 270] = 0.0
    X, info = gpu_call(handle, "trtri", "d", "L", T, "N")
    assert info == O.trtri("d", "L", T.copy(order="F")) == 271
    assert np.array_equal(X, T)    # a singular input is left unmodified
    U = np.asfortranarray(T.T.copy())
    _, info = gpu_call(handle, "trtri", "d", "U", U, "N")
    assert info == O.trtri("d", "U", U.copy(order="F")) == 11


@pytest.mark.parametrize("p", list("sdcz"))
def test_trti22_small_block(handle, p):
    import torch
    n = 40
    A = matgen.spd(p, n, seed=4)
    Fo = A.copy(order="F")
    O.potrf(p, "L", Fo)
    Ta = cc.to_device_colmajor(Fo)
    Tb = torch.zeros_like(Ta)
    dinfo = torch.full((1,), 77, dtype=torch.int32, device="cuda")
    rc = cc.call_trti22(handle, p.upper(), "L", "N", n, Ta.data_ptr(), n, Tb.data_ptr(), n, dinfo.data_ptr())
    assert rc == 0
    torch.cuda.synchronize()
    assert int(dinfo.item()) == 0
    Xo = Fo.copy(order="F")
    O.trtri(p, "L", Xo)
    X = cc.to_host_colmajor(Tb)
    assert np.abs(np.tril(X - Xo)).max() / np.abs(Xo).max() <= 1e3 * n * EPS[p]
    rc = cc.call_trti22(handle, p.upper(), "L", "N", 200, Ta.data_ptr(), n, Tb.data_ptr(), n, dinfo.data_ptr())
    assert rc == cc.CUDA_ERROR_INVALID_VALUE


@pytest.mark.parametrize("p", list("sdcz"))
def test_logdet_vector(handle, p):
    """The reference test's check (test/lapack/dlogdet.c:38-49): a Kahan-summed
    2*sum log x, here with a relative bound of 100*n*eps, contiguous and strided."""
    import torch
    rng = np.random.default_rng(9)
    for n, incx in ((1, 1), (1000, 1), (100000, 1), (5000, 3)):
        x = (rng.uniform(0.0, 1.0, n * incx) + 1e-3).astype(matgen.dtype_of(p))
        T = torch.from_numpy(x).cuda()
        rc, out = cc.call_logdet(handle, p.upper(), T.data_ptr(), incx, n)
        assert rc == 0
        torch.cuda.synchronize()
        s = c = 0.0
        for v in np.log(np.real(x[::incx]).astype(np.float64)):
            y = v - c
            t = s + y
            c = (t - s) - y
            s = t
        ref = 2 * s
        assert abs(out.value - ref) <= 100 * n * EPS[p] * max(1.0, abs(ref)), (n, incx, out.value, ref)


def test_determinism(handle):
    A = matgen.spd("d", 700, seed=2)
    F1, _ = gpu_call(handle, "potrf", "d", "L", A)
    F2, _ = gpu_call(handle, "potrf", "d", "L", A)
    assert np.array_equal(F1, F2)
    X1, _ = gpu_call(handle, "potri", "d", "L", F1)
    X2, _ = gpu_call(handle, "potri", "d", "L", F1)
    assert np.array_equal(X1, X2)


@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("u", ["L", "U"])
def test_outer_block_sizes(handle, p, u):
    """Every ?potrf outer-block size the tuning table accepts (1..16 diagonal
    blocks, here forced per handle) gives a factor within the bounds, on an order
    that leaves a partial outer block and, at the widest blocks, trailing updates
    with k >= 1024 over >= 256 rows (the large-tile FP32 path); the table's own
    choice is restored after."""
    import ctypes as C
    from cucholesky import tune
    lib = cc.lib()
    tune._declare(lib)
    n = 2200
    # lda = n + 3 takes the general engines; for FP32, lda = n (16-byte rows) takes the
    # split TF32 tensor-core updates
    ldas = (n + 3, n) if p == "s" else (n + 3,)
    try:
        for lda in ldas:
            A = matgen.spd(p, n, seed=5, lda=lda)
            Fo = A.copy(order="F")
            assert O.potrf(p, u, Fo, lda=lda) == 0
            for sub in (1, 2, 3, 4, 5, 6, 8, 12, 16):
                assert lib.cuLAPACKSetPotrfBlocks(handle.value, sub) == 0
                F, info = gpu_call(handle, "potrf", p, u, A)
                assert info == 0
                assert matgen.backward_error(A, F, u) <= 10, (lda, sub)
                d = np.abs(_tri(u)(F[:n, :n] - Fo[:n, :n])).max()
                assert d <= 50 * n * EPS[p] * np.abs(A[:n, :n]).max(), (lda, sub, d)
    finally:
        assert lib.cuLAPACKSetPotrfBlocks(handle.value, 0) == 0
    v = C.c_int(0)
    tune_expected = {"d": 5, "z": 12, "s": 4, "c": 6}
    assert lib.cuLAPACKGetPotrfBlocks(handle.value, p.upper().encode(), 16384, C.byref(v)) == 0
    assert v.value == tune_expected[p]


@pytest.mark.parametrize("p", list("sdcz"))
def test_lauum_in_place_block_columns(p):
    """?lauum forms the product one block column at a time in place; a handle whose
    block width is forced small (CUCHOLESKY_LAUUM_COLS, read at handle creation)
    runs several block columns, including a ragged last one."""
    import os
    old = os.environ.get("CUCHOLESKY_LAUUM_COLS")
    os.environ["CUCHOLESKY_LAUUM_COLS"] = "256"
    try:
        h = cc.Handle()
    finally:
        if old is None:
            del os.environ["CUCHOLESKY_LAUUM_COLS"]
        else:
            os.environ["CUCHOLESKY_LAUUM_COLS"] = old
    try:
        for u in "LU":
            n, lda = 700, 703
            A = matgen.spd(p, n, seed=23, lda=lda)
            Fo = A.copy(order="F")
            assert O.potrf(p, u, Fo, lda=lda) == 0
            Lm, _ = gpu_call(h, "lauum", p, u, Fo)
            Lo = Fo.copy(order="F")
            O.lauum(p, u, Lo)          # the oracle takes lda from the array's rows
            d = np.abs(_tri(u)(Lm[:n, :n] - Lo[:n, :n])).max() / np.abs(Lo[:n, :n]).max()
            assert d <= 100 * n * EPS[p], (u, d)
            other = np.triu(np.ones((n, n), bool), 1) if u == "L" else np.tril(np.ones((n, n), bool), -1)
            assert np.array_equal(Lm[:n, :n][other], Fo[:n, :n][other])
            assert np.array_equal(Lm[n:, :], Fo[n:, :])
    finally:
        h.close()
