"""cuDlogdetNoAlloc: the log-determinant entry point for callers that cannot
allocate device memory (its scratch is a static device array, not a handle's
cudaMalloc'd workspace).  Checked through the C ABI against the handle-based
cuDlogdet on the same inputs, twice in a row, since every call reuses the same
static scratch.  This file is collected last on purpose."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import cucholesky as cc
from cucholesky import matgen

pytestmark = pytest.mark.gpu

MAX_N = 8_388_608
EPS = np.finfo(np.float64).eps


def _noalloc():
    f = cc.lib().cuDlogdetNoAlloc
    f.argtypes = [C.c_uint64, C.c_size_t, C.c_size_t, C.POINTER(C.c_double), C.c_void_p]
    f.restype = C.c_int
    return f


def _reference_logdet(handle, ptr, incx, n):
    import torch
    rc, out = cc.call_logdet(handle, "D", ptr, incx, n)
    assert rc == 0
    torch.cuda.synchronize()
    return float(out.value)


def _noalloc_logdet(ptr, incx, n):
    import torch
    out = C.c_double(float("nan"))
    rc = _noalloc()(ptr, incx, n, C.byref(out), None)
    assert rc == 0
    torch.cuda.synchronize()
    return out.value


def test_noalloc_matches_cudlogdet_twice(handle):
    import torch
    rng = np.random.default_rng(17)
    cases = []
    # the diagonal of a Cholesky factor (stride lda + 1), as the path uses it
    n = 700
    A = matgen.spd("d", n, seed=3)
    T = cc.to_device_colmajor(A)
    rc, info = cc.call_potrf(handle, "D", "L", n, T.data_ptr(), n)
    assert rc == 0 and info == 0
    cases.append((T, n + 1, n))
    # contiguous vectors across the chunk boundaries of the static scratch
    for m in (1, 2047, 2048, 2049, 100_000, 1_000_000):
        x = torch.from_numpy(rng.uniform(0.5, 2.0, m)).cuda()
        cases.append((x, 1, m))
    for buf, incx, m in cases:
        ref = _reference_logdet(handle, buf.data_ptr(), incx, m)
        tol = 100 * m * EPS * max(1.0, abs(ref))
        first = _noalloc_logdet(buf.data_ptr(), incx, m)
        second = _noalloc_logdet(buf.data_ptr(), incx, m)
        assert abs(first - ref) <= tol, (m, first, ref)
        assert abs(second - ref) <= tol, (m, second, ref)


def test_noalloc_allocates_nothing_after_first_call():
    """After a first call on the device (which may load the library's kernels), a
    call leaves the device's free memory exactly unchanged: it allocates nothing."""
    import torch
    x = torch.from_numpy(np.random.default_rng(5).uniform(0.5, 2.0, 300_000)).cuda()
    _noalloc_logdet(x.data_ptr(), 1, x.numel())            # warm-up: module load, address lookup
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    out = C.c_double(float("nan"))
    for _ in range(3):
        assert _noalloc()(x.data_ptr(), 1, x.numel(), C.byref(out), None) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert np.isfinite(out.value)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    out = C.c_double(1.0)
    assert _noalloc()(0, 1, MAX_N + 1, C.byref(out), None) == cc.CUDA_ERROR_INVALID_VALUE
    assert _noalloc()(0, 1, 0, C.byref(out), None) == 0 and out.value == 0.0
