"""Parity at the orders the library is measured on (the plain drop-in at n = 16384
for real types and n = 8192 for complex ones, both storages; the mixed solve at
n = 32768; the Ozaki-sliced factor at n = 16384), through the C ABI.

The CPU oracle takes minutes to factor these orders, so a factor is judged by the
contract's bounds computed in FP64 on the device with Gaussian probes (the
estimators are in cucholesky.matgen):
  * backward error  ||A - L L^H||_F / (n eps ||A||_F)          <= 10
  * inverse residual ||I - A inv(A)||_F / (n kappa eps)        <= 10
  * log det: cu?logdet of the factor's diagonal against an FP64 sum of the logs of
    the same diagonal (<= 100 n eps relative), and against the FP64 log det of A
    from an independent FP64 Cholesky (torch), within the bound the perturbation
    by the factor's rounding allows;
  * info bit-exact with the oracle on the variant with A[1000][1000] = -1 (the
    oracle's left-looking factor stops at that column, so it runs in seconds).
This is the reference's own protocol (test/lapack/cudpotrf.c:12-153), gated on
the error bounds instead of on info alone."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O
import cucholesky as cc
from cucholesky import matgen

pytestmark = pytest.mark.gpu

EPS = {"s": 2.0 ** -23, "d": 2.0 ** -52, "c": 2.0 ** -23, "z": 2.0 ** -52}
ORDER = {"d": 16384, "s": 16384, "z": 8192, "c": 8192}


def _free(*ts):
    import torch
    for t in ts:
        del t
    torch.cuda.empty_cache()


@pytest.mark.parametrize("p", list("dzsc"))
@pytest.mark.parametrize("u", ["L", "U"])
def test_potrf_potri_logdet_at_benchmark_order(handle, p, u):
    import torch
    n = ORDER[p]
    A64 = matgen.spd_device(p, n, seed=0)                 # FP64 / complex128, T = M^T
    T = A64.to(matgen.torch_dtype(p))                      # the routine's type
    Aexact = matgen.hermitian_of(T, u)                     # the rounded input, in FP64
    del A64
    torch.cuda.empty_cache()

    rc, info = cc.call_potrf(handle, p.upper(), u, n, T.data_ptr(), n)
    torch.cuda.synchronize()
    assert rc == 0 and info == 0, (rc, info)
    L = matgen.factor_of(T, u)
    be = matgen.probe_backward_error(Aexact, L, p)
    assert be <= 10, (p, u, be)

    # log det: the reduction against FP64 sums of the same diagonal, and the factor
    # against an independent FP64 factor of the same (rounded) input
    rc, ld = cc.call_logdet(handle, p.upper(), T.data_ptr(), n + 1, n)
    torch.cuda.synchronize()
    assert rc == 0
    dg = torch.diagonal(L).real
    ref_same = 2.0 * float(torch.log(dg).sum().item())
    assert abs(ld.value - ref_same) <= 100 * n * EPS[p] * max(1.0, abs(ref_same)), (ld.value, ref_same)
    ref_exact = 2.0 * float(torch.log(torch.diagonal(torch.linalg.cholesky(Aexact)).real).sum().item())
    assert abs(ld.value - ref_exact) <= 100 * n * EPS[p] * max(1.0, abs(ref_exact)), (ld.value, ref_exact)
    del L, dg
    torch.cuda.empty_cache()

    rc, info = cc.call_potri(handle, p.upper(), u, n, T.data_ptr(), n)
    torch.cuda.synchronize()
    assert rc == 0 and info == 0, (rc, info)
    Ainv = matgen.hermitian_of(T, u)
    ir = matgen.probe_inverse_residual(Aexact, Ainv, p)
    assert ir <= 10, (p, u, ir)
    del Ainv, T, Aexact
    torch.cuda.empty_cache()


@pytest.mark.parametrize("p", list("dzsc"))
@pytest.mark.parametrize("u", ["L", "U"])
def test_info_at_benchmark_order(handle, p, u):
    """A[1000][1000] = -1: the first non-positive leading minor is 1001, on the GPU
    and in the oracle (whose left-looking loop stops there)."""
    import torch
    n = ORDER[p]
    T = matgen.spd_device(p, n, seed=3).to(matgen.torch_dtype(p))
    T[1000, 1000] = -1.0
    Ah = np.asfortranarray(T.cpu().numpy().T)             # column-major host copy
    rc, info = cc.call_potrf(handle, p.upper(), u, n, T.data_ptr(), n)
    torch.cuda.synchronize()
    assert rc == 0 and info == 1001, (rc, info)
    assert O.potrf(p, u, Ah) == info
    del T
    torch.cuda.empty_cache()


@pytest.mark.parametrize("u", ["L", "U"])
def test_dpotrf_n16384_is_deterministic_and_leaves_the_other_triangle(handle, u):
    import torch
    n = 16384
    A = matgen.spd_device("d", n, seed=5)
    mark = torch.triu(torch.full((n, n), 7.0, dtype=torch.float64, device="cuda"), 1)
    # T = M^T: M's lower triangle is T's upper one, and M's strict upper (not
    # referenced in lower storage) is T's strict lower, here filled with 7
    T0 = torch.triu(A) + mark.T if u == "L" else torch.tril(A) + mark
    T1, T2 = T0.clone(), T0.clone()
    for T in (T1, T2):
        rc, info = cc.call_potrf(handle, "D", u, n, T.data_ptr(), n)
        assert rc == 0 and info == 0
    torch.cuda.synchronize()
    assert torch.equal(T1, T2)
    other = torch.tril(torch.ones(n, n, dtype=torch.bool, device="cuda"), -1)
    if u == "U":
        other = other.T
    assert torch.equal(T1[other], T0[other])
    del A, mark, T0, T1, T2, other
    torch.cuda.empty_cache()


def _berr_rows(A, X, B):
    """max over right-hand sides of |b - A x|_inf / (|A|_inf |x|_inf + |b|_inf)."""
    import torch
    R = B - X @ A               # rows are right-hand sides (A symmetric)
    anorm = A.abs().sum(dim=1).max().item()
    return max(R[c].abs().max().item() / (anorm * X[c].abs().max().item() + B[c].abs().max().item())
               for c in range(B.shape[0]))


@pytest.mark.parametrize("k", [0.0, 2.0])
def test_mixed_solve_n32768(handle, k):
    """The mixed-precision refined solve at its benchmark order, TF32 and BF16
    trailing updates: the refined solution's normwise backward error meets
    sqrt(n) eps (the solver's stopping rule) and so the contract's 10 n eps."""
    import torch
    n, nrhs = 32768, 16
    A = matgen.scaled_spd_device(n, k, seed=int(k))
    g = torch.Generator(device="cuda")
    g.manual_seed(100 + int(k))
    B = torch.randn((nrhs, n), generator=g, device="cuda", dtype=torch.float64)
    for prec in (cc.MIXED_TF32, cc.MIXED_BF16):
        X = torch.zeros_like(B)
        plan = cc.MixedPlan(handle, "L", n, A.data_ptr(), n, prec)
        assert plan.info == 0
        it, berr = plan.solve(nrhs, B.data_ptr(), n, X.data_ptr(), n)
        plan.close()
        assert it > 0, it
        assert berr <= np.sqrt(n) * EPS["d"], (prec, it, berr)
        be = _berr_rows(A, X, B)
        assert be <= 10 * n * EPS["d"], (prec, be)
        assert be <= 2 * np.sqrt(n) * EPS["d"], (prec, be)
        del X
    del A, B
    torch.cuda.empty_cache()


def test_ozaki_factor_n16384(handle):
    """cuDpotrfOzaki (7 INT8 slices, its default at this order) at n = 16384: the
    contract's backward error, agreement with the native factor, the inverse from
    it, and the info of the non-SPD variant."""
    import torch
    n = 16384
    lib = cc.lib()
    lib.cuDpotrfOzaki.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_uint64, C.c_size_t, C.c_int,
                                  C.POINTER(C.c_long)]
    lib.cuDpotrfOzaki.restype = C.c_int
    A = matgen.spd_device("d", n, seed=8)
    To = A.clone()
    info = C.c_long(0)
    assert lib.cuDpotrfOzaki(handle.value, ord("L"), n, To.data_ptr(), n, 0, C.byref(info)) == 0
    torch.cuda.synchronize()
    assert info.value == 0
    Lo = matgen.factor_of(To, "L")
    be = matgen.probe_backward_error(A, Lo, "d")
    assert be <= 10, be
    Tn = A.clone()
    rc, ninfo = cc.call_potrf(handle, "D", "L", n, Tn.data_ptr(), n)
    torch.cuda.synchronize()
    assert rc == 0 and ninfo == 0
    Ln = matgen.factor_of(Tn, "L")
    d = (Lo - Ln).abs().max().item() / Ln.abs().max().item()
    assert d <= 100 * n * EPS["d"], d
    del Ln, Tn, Lo
    torch.cuda.empty_cache()
    rc, pinfo = cc.call_potri(handle, "D", "L", n, To.data_ptr(), n)
    torch.cuda.synchronize()
    assert rc == 0 and pinfo == 0
    Ainv = matgen.hermitian_of(To, "L")
    ir = matgen.probe_inverse_residual(A, Ainv, "d")
    assert ir <= 10, ir
    del Ainv
    torch.cuda.empty_cache()
    Tb = A.clone()
    Tb[1000, 1000] = -1.0
    assert lib.cuDpotrfOzaki(handle.value, ord("L"), n, Tb.data_ptr(), n, 0, C.byref(info)) == 0
    assert info.value == 1001
    del A, To, Tb
    torch.cuda.empty_cache()
