"""Device RNG (cuRng32 / cuRng64, reference include/rng.h:238-413; Philox4x32-10 here)
against the host restatement in philox_ref.py, bit for bit, and the device SPD
generator cu?latmc (the reference's test generator, test/lapack/util/dlatmc.c:11-70)
against the matrix it must produce: exactly Hermitian, eigenvalues equal to the
diagonal drawn from the same stream, factorable, log det = sum log d."""
from __future__ import annotations

import numpy as np
import pytest

import cucholesky as cc
import philox_ref as P

pytestmark = pytest.mark.gpu


def _dev(n, dtype):
    import torch
    return torch.empty(n, dtype=dtype, device="cuda")


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_rng32_words_and_floats(cuda):
    torch = cuda
    g = cc.Rng(32, seed=0x1234ABCD)
    key = (0x1234ABCD, 0)
    x = _dev(1001, torch.int32)
    assert g.fill(x.data_ptr(), 1001, "raw") == 0
    torch.cuda.synchronize()
    want = P.words(key, 0, 1001)
    assert np.array_equal(x.cpu().numpy().view(np.uint32), want)
    # the next fill starts at the next 128-bit block (word 1004)
    pos = 1004
    for kind in ("oo", "oc", "co", "cc"):
        f = _dev(777, torch.float32)
        assert g.fill(f.data_ptr(), 777, kind) == 0
        torch.cuda.synchronize()
        w = P.words(key, pos, 777)
        assert np.array_equal(f.cpu().numpy(), P.to_f32(w, kind)), kind
        pos += 4 * ((777 + 3) // 4)
        v = f.cpu().numpy()
        assert (v > 0).all() if kind in ("oo", "oc") else (v >= 0).all()
        assert (v < 1).all() if kind in ("oo", "co") else (v <= 1).all()
    # reseeding restarts the stream
    g.set(0x1234ABCD)
    y = _dev(8, torch.int32)
    g.fill(y.data_ptr(), 8)
    torch.cuda.synchronize()
    assert np.array_equal(y.cpu().numpy().view(np.uint32), want[:8])
    g.close()


def test_rng64_integers_and_doubles(cuda):
    torch = cuda
    seed = 0x0123456789ABCDEF
    g = cc.Rng(64, seed=seed)
    key = (seed & 0xFFFFFFFF, seed >> 32)
    x = _dev(999, torch.int64)
    assert g.fill(x.data_ptr(), 999, "raw") == 0
    torch.cuda.synchronize()
    assert np.array_equal(x.cpu().numpy().view(np.uint64), P.u64(key, 0, 999))
    block = 500                                            # ceil(999 / 2)
    for kind in ("oo", "oc", "co", "cc"):
        f = _dev(513, torch.float64)
        assert g.fill(f.data_ptr(), 513, kind) == 0
        torch.cuda.synchronize()
        assert np.array_equal(f.cpu().numpy(), P.to_f64(P.u64(key, block, 513), kind)), kind
        block += (513 + 1) // 2
    g.close()


def test_rng_large_fill_spreads(cuda):
    """A fill much larger than one pass of the grid (grid-stride loop) matches too."""
    torch = cuda
    g = cc.Rng(64, seed=7)
    n = 5_000_001
    f = _dev(n, torch.float64)
    assert g.fill(f.data_ptr(), n, "co") == 0
    torch.cuda.synchronize()
    v = f.cpu().numpy()
    idx = np.array([0, 1, 12345, n // 2, n - 2, n - 1])
    full = P.to_f64(P.u64((7, 0), 0, n), "co")
    assert np.array_equal(v[idx], full[idx])
    assert abs(v.mean() - 0.5) < 1e-3


def _host_diag(prefix, seed, n, c):
    bits = 32 if prefix in "SC" else 64
    draws = (n - 2) + (2 if prefix in "CZ" else 1) * n
    if bits == 32:
        r = P.to_f32(P.words((seed, 0), 0, draws), "cc").astype(np.float64)
    else:
        r = P.to_f64(P.u64((seed & 0xFFFFFFFF, seed >> 32), 0, draws), "cc")
    d = np.concatenate([[1.0, c], r[: n - 2] * (c - 1.0) + 1.0])
    return d


@pytest.mark.parametrize("prefix", list("SDCZ"))
def test_latmc(cuda, handle, prefix):
    torch = cuda
    n, lda, c = 300, 303, 100.0
    dt = {"S": torch.float32, "D": torch.float64, "C": torch.complex64, "Z": torch.complex128}[prefix]
    g = cc.Rng(32 if prefix in "SC" else 64, seed=42)
    T = torch.full((n, lda), 7.0, dtype=dt, device="cuda")            # column-major (lda, n)
    assert cc.call_latmc(prefix, g, n, c, T.data_ptr(), lda) == 0
    torch.cuda.synchronize()
    A = T.cpu().numpy().T                                             # (lda, n)
    assert np.all(A[n:, :] == 7.0)                                    # padding untouched
    M = A[:n, :n].astype(np.complex128 if prefix in "CZ" else np.float64)
    assert np.array_equal(A[:n, :n], A[:n, :n].conj().T)              # exactly Hermitian
    d = np.sort(_host_diag(prefix, 42, n, c))
    ev = np.linalg.eigvalsh(M)
    eps = np.finfo(np.float32 if prefix in "SC" else np.float64).eps
    assert np.abs(ev - d).max() <= 50 * n * eps * c, np.abs(ev - d).max()
    # factorable, and log det A = sum log d
    rc, info = cc.call_potrf(handle, prefix, "L", n, T.data_ptr(), lda)
    assert rc == 0 and info == 0
    rc, ld = cc.call_logdet(handle, prefix, T.data_ptr(), lda + 1, n)
    torch.cuda.synchronize()
    assert abs(ld.value - np.log(d).sum()) <= 100 * n * eps * np.log(d).sum()
    g.close()


def test_latmc_large_condition_and_size(cuda, handle):
    """n = 4096, c = 1e6 in FP64: the factor succeeds and the log det matches."""
    torch = cuda
    n, c = 4096, 1e6
    g = cc.Rng(64, seed=2024)
    T = torch.empty((n, n), dtype=torch.float64, device="cuda")
    assert cc.call_latmc("D", g, n, c, T.data_ptr(), n) == 0
    rc, info = cc.call_potrf(handle, "D", "L", n, T.data_ptr(), n)
    assert rc == 0 and info == 0
    rc, ld = cc.call_logdet(handle, "D", T.data_ptr(), n + 1, n)
    torch.cuda.synchronize()
    want = np.log(_host_diag("D", 2024, n, c)).sum()
    assert abs(ld.value - want) <= 1e-9 * abs(want)
