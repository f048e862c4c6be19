"""Failure paths, made to happen on the host or by a bounded device wait that runs
out (nothing here faults or hangs the GPU):

* an allocation that fails (cuLAPACKFailAllocation): cuLAPACKCreate and the
  workspace growth of a call report CUDA_ERROR_OUT_OF_MEMORY through errorHandler,
  leave nothing behind, and the same handle works on the next call;
* a device wait that gives up (cuLAPACKSetWaitLimit with 0 polls on the ticket
  waits of cu?potrs' triangular solves): the call returns CUDA_ERROR_LAUNCH_TIMEOUT
  through errorHandler, and the next call on the same handle, with the default
  limit, gives the right solution.
The convention is the reference's: a CUresult per call and the errorHandler
callback (include/error.h:42-65, multigpu/error.c:4-11)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O
import cucholesky as cc
from cucholesky import matgen

pytestmark = pytest.mark.gpu

CUDA_ERROR_OUT_OF_MEMORY = 2
CUDA_ERROR_LAUNCH_TIMEOUT = 702
HANDLER = C.CFUNCTYPE(None, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_void_p)


class ErrorHandler:
    """Installs a recording errorHandler for the duration of a with-block."""

    def __enter__(self):
        self.calls = []
        self.cb = HANDLER(lambda call, fn, file, line, err, strerr: self.calls.append((call.decode(), err)))
        self.slot = C.c_void_p.in_dll(cc.lib(), "errorHandler")
        self.old = self.slot.value
        self.slot.value = C.cast(self.cb, C.c_void_p).value
        return self

    def __exit__(self, *exc):
        self.slot.value = self.old


def _lib():
    L = cc.lib()
    L.cuLAPACKFailAllocation.argtypes = [C.c_int]
    L.cuLAPACKFailAllocation.restype = C.c_int
    L.cuLAPACKSetWaitLimit.argtypes = [C.c_void_p, C.c_int]
    L.cuLAPACKSetWaitLimit.restype = C.c_int
    L.cuLAPACKCreate.argtypes = [C.POINTER(C.c_void_p)]
    L.cuLAPACKCreate.restype = C.c_int
    return L


def test_create_reports_out_of_memory_and_recovers():
    import torch
    L = _lib()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    with ErrorHandler() as eh:
        # the first, a middle and the last device allocation of a handle fail; the
        # creation frees what it allocated before the failure
        for after in (0, 2, 5):
            assert L.cuLAPACKFailAllocation(after) == 0
            h = C.c_void_p()
            assert L.cuLAPACKCreate(C.byref(h)) == CUDA_ERROR_OUT_OF_MEMORY, after
        assert L.cuLAPACKFailAllocation(-1) == 0
        assert sum(1 for _, e in eh.calls if e == CUDA_ERROR_OUT_OF_MEMORY) == 3
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 >= free0 - (64 << 20), (free0, free1)     # nothing left allocated (allocator slack)
    h = cc.Handle()                                  # allocations work again
    A = matgen.spd("d", 100, seed=1)
    T = cc.to_device_colmajor(A)
    rc, info = cc.call_potrf(h, "D", "L", 100, T.data_ptr(), 100)
    assert rc == 0 and info == 0
    h.close()


def test_workspace_growth_out_of_memory_leaves_handle_usable():
    import torch
    L = _lib()
    h = cc.Handle()
    n = 1500
    A = matgen.spd("d", n, seed=2)
    Fo = A.copy(order="F")
    assert O.potrf("d", "L", Fo) == 0
    with ErrorHandler() as eh:
        T = cc.to_device_colmajor(A)
        assert L.cuLAPACKFailAllocation(0) == 0           # the handle's first workspace
        rc, info = cc.call_potrf(h, "D", "L", n, T.data_ptr(), n)
        assert L.cuLAPACKFailAllocation(-1) == 0
        assert rc == CUDA_ERROR_OUT_OF_MEMORY
        assert eh.calls and eh.calls[-1][1] == CUDA_ERROR_OUT_OF_MEMORY
    torch.cuda.synchronize()
    T = cc.to_device_colmajor(A)
    rc, info = cc.call_potrf(h, "D", "L", n, T.data_ptr(), n)
    assert rc == 0 and info == 0
    F = cc.to_host_colmajor(T)
    assert matgen.backward_error(A, F, "L") <= 10
    assert np.abs(np.tril(F - Fo)).max() <= 50 * n * np.finfo(float).eps * np.abs(A).max()
    h.close()


def test_triangular_solve_wait_timeout_then_recovery():
    import torch
    L = _lib()
    h = cc.Handle()
    n, nrhs = 700, 3                                  # 11 row blocks: every block but the first waits
    A = matgen.spd("d", n, seed=4)
    F = A.copy(order="F")
    assert O.potrf("d", "L", F) == 0
    TF = cc.to_device_colmajor(F)
    rhs = np.random.default_rng(4).standard_normal((n, nrhs))
    with ErrorHandler() as eh:
        assert L.cuLAPACKSetWaitLimit(h.value, 0) == 0
        TB = torch.from_numpy(np.ascontiguousarray(rhs.T)).cuda()
        rc, info = cc.call_potrs(h, "D", "L", n, nrhs, TF.data_ptr(), n, TB.data_ptr(), n)
        assert rc == CUDA_ERROR_LAUNCH_TIMEOUT, rc
        assert any(e == CUDA_ERROR_LAUNCH_TIMEOUT for _, e in eh.calls)
    assert L.cuLAPACKSetWaitLimit(h.value, -1) == 0       # the default limit again
    TB = torch.from_numpy(np.ascontiguousarray(rhs.T)).cuda()
    rc, info = cc.call_potrs(h, "D", "L", n, nrhs, TF.data_ptr(), n, TB.data_ptr(), n)
    torch.cuda.synchronize()
    assert rc == 0 and info == 0
    X = TB.cpu().numpy().T
    Lf = np.tril(F)
    Xref = np.linalg.solve(Lf.T, np.linalg.solve(Lf, rhs))
    assert np.abs(X - Xref).max() <= 1e-10 * np.abs(Xref).max()
    h.close()
