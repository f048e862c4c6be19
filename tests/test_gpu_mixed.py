"""The mixed-precision SPD solve and ?potrs through the C ABI.

* cu?potrs (FP64 and FP32, both storages, ragged n, several groups of right-hand
  sides) against the FP64 solve of the same matrix, with the backward error bound
  of the contract (<= 10 n eps).
* cuDcholMixedCreate: the FP32 factor of S A S + shift I built with BF16 or TF32
  tensor-core trailing updates reproduces S A S + shift I to the operand precision.
* cuDcholMixedSolve / cuDposvMixed: FP64 refinement reaches the FP64 backward error
  (<= sqrt(n) eps, far below the contract's 10 n eps) on the scaled family
  A = D (G G^T / n + 1e-3 I) D for kappa up to ~1e9, and the solution matches the
  FP64 oracle's within kappa * berr; non-SPD input falls back to FP64 with the
  oracle's info."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import cucholesky as cc
from cucholesky import matgen

pytestmark = pytest.mark.gpu

EPS64 = np.finfo(np.float64).eps


def _dev(A):
    import torch
    return torch.from_numpy(np.asfortranarray(A).T.copy()).cuda()   # (cols, rows): column-major


def _host(T):
    return T.cpu().numpy().T


def _oracle_solve(A, B):
    """FP64 solution from the oracle's factor (the reference's dpotrf restated)."""
    from scipy.linalg import solve_triangular
    F = np.asfortranarray(A.copy())
    assert O.potrf("d", "L", F) == 0
    L = np.tril(F)
    return solve_triangular(L.T, solve_triangular(L, B, lower=True), lower=False)


def _berr(A, X, B):
    R = B - A @ X
    an = np.abs(A).sum(axis=1).max()
    return max(np.abs(R[:, c]).max() / (an * np.abs(X[:, c]).max() + np.abs(B[:, c]).max())
               for c in range(B.shape[1]))


@pytest.mark.parametrize("p", ["d", "s"])
@pytest.mark.parametrize("u", ["L", "U"])
@pytest.mark.parametrize("n,nrhs", [(1, 1), (63, 3), (64, 16), (65, 17), (300, 37), (1000, 16)])
def test_potrs(handle, p, u, n, nrhs):
    import torch
    dt = np.float64 if p == "d" else np.float32
    A = matgen.spd("d", n, seed=n)
    rng = np.random.default_rng(n + 1)
    B = rng.standard_normal((n, nrhs))
    TA = _dev(A.astype(dt))
    rc, info = cc.call_potrf(handle, p.upper(), u, n, TA.data_ptr(), n)
    assert rc == 0 and info == 0
    TB = _dev(B.astype(dt))
    rc, info = cc.call_potrs(handle, p.upper(), u, n, nrhs, TA.data_ptr(), n, TB.data_ptr(), n)
    assert rc == 0 and info == 0
    torch.cuda.synchronize()
    X = _host(TB).astype(np.float64)
    eps = np.finfo(dt).eps
    assert _berr(A, X, B) <= 10 * n * eps
    Xref = _oracle_solve(A, B)
    kappa = np.linalg.cond(A)
    assert np.abs(X - Xref).max() / np.abs(Xref).max() <= 10 * n * eps * kappa


def test_potrs_argument_errors(handle):
    rc, info = cc.call_potrs(handle, "D", "L", 10, 1, 0, 10, 0, 5)
    assert rc == cc.CUDA_ERROR_INVALID_VALUE and info == -8
    rc, info = cc.call_potrs(handle, "D", "X", 10, 1, 0, 10, 0, 10)
    assert rc == cc.CUDA_ERROR_INVALID_VALUE and info == -2


@pytest.mark.parametrize("prec,bound", [(cc.MIXED_BF16, 3e-2), (cc.MIXED_TF32, 4e-3)])
@pytest.mark.parametrize("n", [200, 777, 1536])
def test_mixed_factor_accuracy(handle, prec, bound, n):
    """W W^T reproduces S A S + shift I to the operand precision (relative
    Frobenius error; FP32 factor, BF16 / TF32 trailing products)."""
    import torch
    A = matgen.scaled_spd(n, 2.0, seed=n)
    TA = _dev(A)
    plan = cc.MixedPlan(handle, "L", n, TA.data_ptr(), n, prec)
    assert plan.info == 0
    w, ldw, s, anorm, shift = plan.factor()
    torch.cuda.synchronize()
    plan_w = _copy_device(w, n * ldw, torch.float32).reshape(n, ldw)
    S = _copy_device(s, n, torch.float64).cpu().numpy()
    Wh = plan_w.cpu().numpy().T[:n, :n]
    L = np.tril(np.where(np.tril(np.ones((n, n), dtype=bool)), Wh, 0.0).astype(np.float64))
    H = S[:, None] * A * S[None, :] + shift * np.eye(n)
    err = np.linalg.norm(H - L @ L.T) / np.linalg.norm(H)
    assert err <= bound, err
    assert abs(anorm - np.abs(A).sum(axis=1).max()) <= 1e-12 * anorm
    plan.close()


def _copy_device(ptr, count, dtype):
    """Copy `count` elements at a raw device address into a new torch tensor
    (zero-copy view through __cuda_array_interface__, then a clone)."""
    import torch

    class _Raw:
        __cuda_array_interface__ = {"shape": (count,), "typestr": "<f4" if dtype == torch.float32 else "<f8",
                                    "data": (ptr, False), "version": 2}

    return torch.as_tensor(_Raw(), device="cuda").clone()


@pytest.mark.parametrize("prec", [cc.MIXED_BF16, cc.MIXED_TF32])
@pytest.mark.parametrize("k", [0, 1, 3])
@pytest.mark.parametrize("u", ["L", "U"])
def test_mixed_solve(handle, prec, k, u):
    import torch
    n, nrhs = 1000, 16
    A = matgen.scaled_spd(n, float(k), seed=7 + k)
    rng = np.random.default_rng(11)
    B = rng.standard_normal((n, nrhs))
    Astore = np.tril(A) if u == "L" else np.triu(A)   # only one triangle is referenced
    TA = _dev(Astore + (np.triu(np.full((n, n), np.nan), 1) if u == "L" else np.tril(np.full((n, n), np.nan), -1)))
    TB, TX = _dev(B), _dev(np.zeros_like(B))
    plan = cc.MixedPlan(handle, u, n, TA.data_ptr(), n, prec)
    assert plan.info == 0
    it, berr = plan.solve(nrhs, TB.data_ptr(), n, TX.data_ptr(), n)
    torch.cuda.synchronize()
    assert it > 0, (it, berr)
    X = _host(TX)
    tol = np.sqrt(n) * 2.0 ** -53
    assert berr <= tol
    assert _berr(A, X, B) <= 2 * tol            # recomputed on the host in FP64
    assert _berr(A, X, B) <= 10 * n * EPS64     # the contract's bound
    Xref = _oracle_solve(A, B)
    kappa = np.linalg.cond(A)
    assert np.abs(X - Xref).max() / np.abs(Xref).max() <= 100 * kappa * tol
    plan.close()


@pytest.mark.parametrize("n,nrhs", [(129, 1), (257, 20)])
def test_posv_mixed_ragged(handle, n, nrhs):
    import torch
    A = matgen.scaled_spd(n, 1.0, seed=n)
    B = np.random.default_rng(n).standard_normal((n, nrhs))
    TA, TB, TX = _dev(A), _dev(B), _dev(np.zeros_like(B))
    rc, it, berr, info = cc.call_posv_mixed(handle, "L", n, nrhs, TA.data_ptr(), n, TB.data_ptr(), n,
                                            TX.data_ptr(), n, cc.MIXED_TF32)
    torch.cuda.synchronize()
    assert rc == 0 and info == 0 and it > 0
    assert _berr(A, _host(TX), B) <= np.sqrt(n) * 2.0 ** -52
    assert np.array_equal(_host(TA), A)   # A unchanged on the mixed path


def test_posv_mixed_not_spd_falls_back(handle):
    """A non-positive leading minor: the FP64 fallback factors A and reports the
    oracle's info (first failing column), DSPOSV's iter = -3."""
    import torch
    n = 300
    A = matgen.spd("d", n, seed=3)
    A[100, 100] = -1.0
    info_ref = O.potrf("d", "L", A.copy(order="F"))
    B = np.ones((n, 2))
    TA, TB, TX = _dev(A), _dev(B), _dev(np.zeros_like(B))
    rc, it, berr, info = cc.call_posv_mixed(handle, "L", n, 2, TA.data_ptr(), n, TB.data_ptr(), n, TX.data_ptr(),
                                            n, cc.MIXED_BF16)
    torch.cuda.synchronize()
    assert rc == 0 and it == -3
    assert info == info_ref == 101


@pytest.mark.parametrize("prec", [cc.MIXED_BF16, cc.MIXED_TF32])
@pytest.mark.parametrize("n,k", [(1, 8), (127, 64), (300, 200), (1024, 512)])
def test_syrk_lowp(handle, prec, n, k):
    """cuSsyrkLowp (the tcgen05 trailing-update kernel) against an FP64 product of
    the same rounded operands: lower triangle updated, upper triangle untouched."""
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(n * 7 + k)
    ldq = (k + 7) // 8 * 8 if prec == cc.MIXED_BF16 else (k + 3) // 4 * 4
    Q32 = torch.rand((n, ldq), generator=g, device="cuda", dtype=torch.float32) * 2 - 1
    if prec == cc.MIXED_BF16:
        Q = Q32.to(torch.bfloat16)
        Qd = Q.double()[:, :k]
    else:
        # TF32 operands: values already representable, so rounding mode does not matter
        Q = (Q32.view(torch.int32) & ~0x1FFF).view(torch.float32)
        Qd = Q.double()[:, :k]
    ldc = (n + 3) // 4 * 4
    Cm = torch.rand((n, ldc), generator=g, device="cuda", dtype=torch.float32)   # column j = row j of Cm
    C0 = Cm.clone()
    rc = cc.call_syrk_lowp(handle, prec, n, k, -1.0, Q.data_ptr(), ldq, Cm.data_ptr(), ldc)
    torch.cuda.synchronize()
    assert rc == 0
    ref = C0.double()[:, :n].T - Qd @ Qd.T        # column-major C as a (n, n) matrix
    got = Cm.double()[:, :n].T
    low = torch.tril(torch.ones(n, n, dtype=torch.bool, device="cuda"))
    # FP32 accumulation of k exact products, then one FP32 add to C:
    # |err| <= gamma_{k+1} (|Q||Q|^T + |C|), gamma_j = j u / (1 - j u), u = 2^-24
    u = 2.0 ** -24
    gamma = (k + 1) * u / (1 - (k + 1) * u)
    bound = gamma * (Qd.abs() @ Qd.abs().T + C0.double()[:, :n].T.abs())
    assert bool(((got - ref).abs() <= bound)[low].all()), ((got - ref).abs() - bound)[low].max().item()
    assert torch.equal(got[~low], C0.double()[:, :n].T[~low])
