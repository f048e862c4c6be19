"""Python binding of libcucholesky.so, the sm_100a implementation of the dense SPD
path (?POTRF, ?TRTRI, ?TRTI22, ?LAUUM, ?POTRI, ?LOGDET) behind the C API of
``include/lapack.h``.

The binding is a thin ctypes layer over that C ABI: every call goes through the
exported ``cu?potrf`` / ``cu?potri`` / ... symbols with raw device pointers, the
way a C caller of the reference library would call them.  Device memory comes
from torch tensors (plumbing only).  There is no CPU fallback: if the shared
library is missing, importing the binding's functions raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcucholesky.so")

CUDA_SUCCESS = 0
CUDA_ERROR_INVALID_VALUE = 1

PREFIX = {"float32": "S", "float64": "D", "complex64": "C", "complex128": "Z"}

_lib = None


class CuCholeskyError(RuntimeError):
    def __init__(self, name: str, code: int):
        super().__init__(f"{name} returned CUresult {code}")
        self.code = code


def lib() -> C.CDLL:
    """Load libcucholesky.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `make -C cuda-cholesky_b200/csrc` "
                "(or __graft_entry__.build()); there is no fallback implementation")
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L: C.CDLL) -> None:
    H = C.c_void_p
    for p in "SDCZ":
        for name in ("potrf", "lauum", "potri"):
            f = getattr(L, f"cu{p}{name}")
            f.argtypes = [H, C.c_int, C.c_size_t, C.c_uint64, C.c_size_t, C.POINTER(C.c_long)]
            f.restype = C.c_int
        f = getattr(L, f"cu{p}trtri")
        f.argtypes = [H, C.c_int, C.c_int, C.c_size_t, C.c_uint64, C.c_size_t, C.POINTER(C.c_long)]
        f.restype = C.c_int
        f = getattr(L, f"cu{p}trti22")
        f.argtypes = [H, C.c_int, C.c_int, C.c_size_t, C.c_uint64, C.c_size_t, C.c_uint64, C.c_size_t,
                      C.c_uint64, C.c_void_p]
        f.restype = C.c_int
        f = getattr(L, f"cu{p}logdet")
        out = C.c_float if p in "SC" else C.c_double
        f.argtypes = [H, C.c_uint64, C.c_size_t, C.c_size_t, C.POINTER(out), C.c_void_p]
        f.restype = C.c_int
    L.cuLAPACKCreate.argtypes = [C.POINTER(C.c_void_p)]
    L.cuLAPACKCreate.restype = C.c_int
    L.cuLAPACKDestroy.argtypes = [C.c_void_p]
    L.cuLAPACKDestroy.restype = C.c_int


def exported_symbols() -> list[str]:
    """Names a C caller links against (the include/lapack.h prototypes)."""
    names = ["cuLAPACKCreate", "cuLAPACKDestroy", "xerbla", "errorHandler", "cuBLASCreate", "cuBLASDestroy",
             "cuSsyrk", "cuDsyrk", "cuCherk", "cuZherk"]
    for p in "SDCZ":
        names += [f"cu{p}{r}" for r in ("potrf", "trtri", "trti22", "lauum", "potri", "logdet", "gemm2", "trsm",
                                         "trmm2")]
        names += [f"cuMultiGPU{p}{r}" for r in ("potrf", "trtri", "lauum", "potri")]
    names += ["cuMultiGPUCreate", "cuMultiGPUDestroy", "cuMultiGPUGetContextCount", "cuMultiGPUSynchronize",
              "cuMultiGPULAPACKCreate", "cuMultiGPULAPACKDestroy", "cuMultiGPULAPACKSynchronize"]
    return names


def extension_symbols() -> list[str]:
    """Entry points of include/cucholesky_ext.h (no counterpart in the reference)."""
    names = [f"cu{p}potrfLogdet" for p in "SDCZ"]
    names += ["cuLAPACKGetLaunchCount", "cuDcholBatchedCreate", "cuScholBatchedCreate", "cuCholBatchedRun",
              "cuCholBatchedResults", "cuCholBatchedGetBlockSize", "cuCholBatchedDestroy", "cuDlogdetNoAlloc",
              "cuDpotrs", "cuSpotrs", "cuDcholMixedCreate", "cuDcholMixedRefactor", "cuDcholMixedSolve",
              "cuCholMixedGetFactor", "cuSsyrkLowp", "cuDpotrfOzaki",
              "cuCholMixedDestroy", "cuDposvMixed", "cuMultiGPULAPACKGetStats", "cuSlatmc", "cuDlatmc", "cuClatmc",
              "cuZlatmc", "philox32_t", "philox64_t", "cuLAPACKFailAllocation", "cuLAPACKSetWaitLimit"]
    for b in ("32", "64"):
        names += [f"cuRng{b}{f}" for f in ("Create", "Destroy", "Set", "Get", "GetOpenOpen", "GetOpenClose",
                                           "GetCloseOpen", "GetCloseClose")]
    return names


class Handle:
    """CULAPACKhandle bound to the current CUDA device."""

    def __init__(self):
        self._h = C.c_void_p()
        rc = lib().cuLAPACKCreate(C.byref(self._h))
        if rc != CUDA_SUCCESS:
            raise CuCholeskyError("cuLAPACKCreate", rc)

    @property
    def value(self) -> C.c_void_p:
        return self._h

    def close(self) -> None:
        if self._h:
            lib().cuLAPACKDestroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _uplo(u: str) -> int:
    return ord(u.upper())


def _prefix(t) -> str:
    return PREFIX[str(t.dtype).replace("torch.", "")]


def _lda(A) -> int:
    """Column-major device matrix as a torch tensor of shape (n_cols, lda) in
    row-major torch terms, i.e. A.T is the (lda, n) column-major matrix."""
    return A.shape[1]


# ---- raw C-ABI calls ------------------------------------------------------------

def call_potrf(h: Handle, prefix: str, uplo: str, n: int, ptr: int, lda: int) -> tuple[int, int]:
    info = C.c_long(0)
    rc = getattr(lib(), f"cu{prefix}potrf")(h.value, _uplo(uplo), n, ptr, lda, C.byref(info))
    return rc, info.value


def call_potri(h: Handle, prefix: str, uplo: str, n: int, ptr: int, lda: int) -> tuple[int, int]:
    info = C.c_long(0)
    rc = getattr(lib(), f"cu{prefix}potri")(h.value, _uplo(uplo), n, ptr, lda, C.byref(info))
    return rc, info.value


def call_lauum(h: Handle, prefix: str, uplo: str, n: int, ptr: int, lda: int) -> tuple[int, int]:
    info = C.c_long(0)
    rc = getattr(lib(), f"cu{prefix}lauum")(h.value, _uplo(uplo), n, ptr, lda, C.byref(info))
    return rc, info.value


def call_trtri(h: Handle, prefix: str, uplo: str, diag: str, n: int, ptr: int, lda: int) -> tuple[int, int]:
    info = C.c_long(0)
    rc = getattr(lib(), f"cu{prefix}trtri")(h.value, _uplo(uplo), _uplo(diag), n, ptr, lda, C.byref(info))
    return rc, info.value


def call_trti22(h: Handle, prefix: str, uplo: str, diag: str, n: int, a: int, lda: int, b: int, ldb: int,
                dinfo: int, stream: int = 0) -> int:
    return getattr(lib(), f"cu{prefix}trti22")(h.value, _uplo(uplo), _uplo(diag), n, a, lda, b, ldb, dinfo,
                                               C.c_void_p(stream))


def call_logdet(h: Handle, prefix: str, ptr: int, incx: int, n: int, stream: int = 0) -> tuple[int, float]:
    out = (C.c_float if prefix in "SC" else C.c_double)(0)
    rc = getattr(lib(), f"cu{prefix}logdet")(h.value, ptr, incx, n, C.byref(out), C.c_void_p(stream))
    return rc, out


# ---- torch conveniences (column-major matrices as transposed torch tensors) ------

def to_device_colmajor(A_np, device="cuda"):
    """numpy (lda, n) Fortran-order array -> torch tensor T of shape (n, lda) whose
    row j is column j of A, i.e. the same bytes as the column-major matrix."""
    import numpy as np
    import torch
    return torch.from_numpy(np.ascontiguousarray(A_np.T)).to(device)


def to_host_colmajor(T):
    import numpy as np
    return np.asfortranarray(T.cpu().numpy().T)


def potrf(h: Handle, T, n: int, uplo: str = "L") -> int:
    rc, info = call_potrf(h, _prefix(T), uplo, n, T.data_ptr(), T.shape[1])
    if rc != CUDA_SUCCESS:
        raise CuCholeskyError(f"cu{_prefix(T)}potrf", rc)
    return info


def potri(h: Handle, T, n: int, uplo: str = "L") -> int:
    rc, info = call_potri(h, _prefix(T), uplo, n, T.data_ptr(), T.shape[1])
    if rc != CUDA_SUCCESS:
        raise CuCholeskyError(f"cu{_prefix(T)}potri", rc)
    return info


def trtri(h: Handle, T, n: int, uplo: str = "L", diag: str = "N") -> int:
    rc, info = call_trtri(h, _prefix(T), uplo, diag, n, T.data_ptr(), T.shape[1])
    if rc != CUDA_SUCCESS:
        raise CuCholeskyError(f"cu{_prefix(T)}trtri", rc)
    return info


def lauum(h: Handle, T, n: int, uplo: str = "L") -> int:
    rc, info = call_lauum(h, _prefix(T), uplo, n, T.data_ptr(), T.shape[1])
    if rc != CUDA_SUCCESS:
        raise CuCholeskyError(f"cu{_prefix(T)}lauum", rc)
    return info


def logdet_of_factor(h: Handle, T, n: int) -> float:
    """log det A from the factor in T (diagonal stride lda + 1), synchronising the
    default stream before returning."""
    import torch
    lda = T.shape[1]
    rc, out = call_logdet(h, _prefix(T), T.data_ptr(), lda + 1, n, 0)
    if rc != CUDA_SUCCESS:
        raise CuCholeskyError(f"cu{_prefix(T)}logdet", rc)
    torch.cuda.synchronize()
    return float(out.value)


# ---- BLAS layer (include/blas.h) -------------------------------------------------

class _CF(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float)]


class _CD(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double)]


_SCAL = {"S": C.c_float, "D": C.c_double, "C": _CF, "Z": _CD}
_REAL = {"S": C.c_float, "D": C.c_double, "C": C.c_float, "Z": C.c_double}


def _declare_blas(L: C.CDLL) -> None:
    L.cuBLASCreate.argtypes = [C.POINTER(C.c_void_p)]
    L.cuBLASCreate.restype = C.c_int
    L.cuBLASDestroy.argtypes = [C.c_void_p]
    L.cuBLASDestroy.restype = C.c_int
    for p in "SDCZ":
        f = getattr(L, f"cu{p}gemm2")
        S = _SCAL[p]
        f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_size_t, C.c_size_t, C.c_size_t, S, C.c_uint64, C.c_size_t,
                      C.c_uint64, C.c_size_t, S, C.c_uint64, C.c_size_t, C.c_uint64, C.c_size_t, C.c_void_p]
        f.restype = C.c_int
    for p in "SDCZ":
        S = _SCAL[p]
        f = getattr(L, f"cu{p}trsm")
        f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_size_t, C.c_size_t, S, C.c_uint64,
                      C.c_size_t, C.c_uint64, C.c_size_t, C.c_void_p]
        f.restype = C.c_int
        f = getattr(L, f"cu{p}trmm2")
        f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_size_t, C.c_size_t, S, C.c_uint64,
                      C.c_size_t, C.c_uint64, C.c_size_t, C.c_uint64, C.c_size_t, C.c_void_p]
        f.restype = C.c_int
    for name, p in (("cuSsyrk", "S"), ("cuDsyrk", "D"), ("cuCherk", "C"), ("cuZherk", "Z")):
        f = getattr(L, name)
        R = _REAL[p]
        f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_size_t, C.c_size_t, R, C.c_uint64, C.c_size_t, R,
                      C.c_uint64, C.c_size_t, C.c_void_p]
        f.restype = C.c_int


class BlasHandle:
    """CUBLAShandle of this library (not NVIDIA cuBLAS)."""

    def __init__(self):
        L = lib()
        if not getattr(L, "_blas_declared", False):
            _declare_blas(L)
            L._blas_declared = True
        self._h = C.c_void_p()
        rc = L.cuBLASCreate(C.byref(self._h))
        if rc != CUDA_SUCCESS:
            raise CuCholeskyError("cuBLASCreate", rc)

    @property
    def value(self):
        return self._h

    def close(self):
        if self._h:
            lib().cuBLASDestroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _scal(p: str, v):
    if p in "CZ":
        v = complex(v)
        return _SCAL[p](v.real, v.imag)
    return _SCAL[p](v)


def call_gemm2(bh: BlasHandle, p: str, ta: str, tb: str, m: int, n: int, k: int, alpha, a: int, lda: int,
               b: int, ldb: int, beta, c: int, ldc: int, d: int, ldd: int, stream: int = 0) -> int:
    return getattr(lib(), f"cu{p}gemm2")(bh.value, ord(ta), ord(tb), m, n, k, _scal(p, alpha), a, lda, b, ldb,
                                         _scal(p, beta), c, ldc, d, ldd, C.c_void_p(stream))


def call_trsm(bh: BlasHandle, p: str, side: str, uplo: str, trans: str, diag: str, m: int, n: int, alpha,
              a: int, lda: int, b: int, ldb: int, stream: int = 0) -> int:
    """cu?trsm: B := alpha op(A)^-1 B (side L) or alpha B op(A)^-1 (side R), in place."""
    return getattr(lib(), f"cu{p}trsm")(bh.value, ord(side), ord(uplo), ord(trans), ord(diag), m, n,
                                        _scal(p, alpha), a, lda, b, ldb, C.c_void_p(stream))


def call_trmm2(bh: BlasHandle, p: str, side: str, uplo: str, trans: str, diag: str, m: int, n: int, alpha,
               a: int, lda: int, b: int, ldb: int, x: int, ldx: int, stream: int = 0) -> int:
    """cu?trmm2: X := alpha op(A) B (side L) or alpha B op(A) (side R)."""
    return getattr(lib(), f"cu{p}trmm2")(bh.value, ord(side), ord(uplo), ord(trans), ord(diag), m, n,
                                         _scal(p, alpha), a, lda, b, ldb, x, ldx, C.c_void_p(stream))


def call_rankk(bh: BlasHandle, p: str, uplo: str, trans: str, n: int, k: int, alpha: float, a: int, lda: int,
               beta: float, c: int, ldc: int, stream: int = 0) -> int:
    name = {"S": "cuSsyrk", "D": "cuDsyrk", "C": "cuCherk", "Z": "cuZherk"}[p]
    return getattr(lib(), name)(bh.value, ord(uplo), ord(trans), n, k, _REAL[p](alpha), a, lda, _REAL[p](beta),
                                c, ldc, C.c_void_p(stream))


# ---- batched plan (include/cucholesky_ext.h) -------------------------------------

BATCHED_POTRF, BATCHED_LOGDET, BATCHED_POTRI = 1, 2, 4


class BatchedPlan:
    """cu?cholBatchedCreate / Run / Results / Destroy for matrices packed in one
    device buffer: matrix b is column-major n[b] x n[b] with leading dimension
    lda[b], starting at element offset off[b] of `buf` (a torch tensor)."""

    def __init__(self, h: Handle, buf, n, off, lda=None, uplo="L", flags=7, nb=0):
        L = lib()
        p = "D" if str(buf.dtype) == "torch.float64" else "S"
        esize = buf.element_size()
        self.batch = len(n)
        lda = list(n) if lda is None else list(lda)
        self._n = (C.c_int * self.batch)(*n)
        self._lda = (C.c_int * self.batch)(*lda)
        base = buf.data_ptr()
        self._ptrs = (C.c_uint64 * self.batch)(*[base + int(o) * esize for o in off])
        self._p = C.c_void_p()
        f = getattr(L, f"cu{p}cholBatchedCreate")
        f.argtypes = [C.POINTER(C.c_void_p), C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int),
                      C.POINTER(C.c_uint64), C.POINTER(C.c_int), C.c_int, C.c_int]
        f.restype = C.c_int
        rc = f(C.byref(self._p), h.value, ord(uplo), self.batch, self._n, self._ptrs, self._lda, flags, nb)
        if rc != CUDA_SUCCESS:
            raise CuCholeskyError(f"cu{p}cholBatchedCreate", rc)
        L.cuCholBatchedRun.argtypes = [C.c_void_p, C.c_void_p]
        L.cuCholBatchedResults.argtypes = [C.c_void_p, C.POINTER(C.c_long), C.POINTER(C.c_double)]
        L.cuCholBatchedGetBlockSize.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        L.cuCholBatchedDestroy.argtypes = [C.c_void_p]

    @property
    def nb(self) -> int:
        v = C.c_int(0)
        lib().cuCholBatchedGetBlockSize(self._p, C.byref(v))
        return v.value

    def run(self, stream: int = 0) -> None:
        rc = lib().cuCholBatchedRun(self._p, C.c_void_p(stream))
        if rc != CUDA_SUCCESS:
            raise CuCholeskyError("cuCholBatchedRun", rc)

    def results(self):
        info = (C.c_long * self.batch)()
        ld = (C.c_double * self.batch)()
        rc = lib().cuCholBatchedResults(self._p, info, ld)
        if rc != CUDA_SUCCESS:
            raise CuCholeskyError("cuCholBatchedResults", rc)
        return list(info), list(ld)

    def close(self):
        if self._p:
            lib().cuCholBatchedDestroy(self._p)
            self._p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pack_colmajor(mats, dtype):
    """Pack square column-major numpy matrices into one 1-D array; returns
    (array, offsets, sizes)."""
    import numpy as np
    sizes = [m.shape[1] for m in mats]
    off, t = [], 0
    for m in mats:
        off.append(t)
        t += m.shape[0] * m.shape[1]
    out = np.zeros(max(t, 1), dtype=dtype)
    for m, o in zip(mats, off):
        out[o:o + m.size] = np.asarray(m, dtype=dtype).ravel(order="F")
    return out, off, sizes


# ---- ?potrs and the mixed-precision solve (include/cucholesky_ext.h) -----------

MIXED_BF16, MIXED_TF32 = 1, 2


def call_potrs(h: Handle, prefix: str, uplo: str, n: int, nrhs: int, a: int, lda: int, b: int,
               ldb: int) -> tuple[int, int]:
    f = getattr(lib(), f"cu{prefix}potrs")
    f.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_size_t, C.c_uint64, C.c_size_t, C.c_uint64, C.c_size_t,
                  C.POINTER(C.c_long)]
    f.restype = C.c_int
    info = C.c_long(0)
    rc = f(h.value, _uplo(uplo), n, nrhs, a, lda, b, ldb, C.byref(info))
    return rc, info.value


class MixedPlan:
    """cuDcholMixedCreate / Solve / GetFactor / Destroy on an FP64 device matrix
    (column-major, leading dimension lda, pointer `a`).  The plan reads A again in
    every solve: keep it unchanged while the plan lives."""

    def __init__(self, h: Handle, uplo: str, n: int, a: int, lda: int, precision: int = MIXED_TF32,
                 shift: float = -1.0):
        L = lib()
        L.cuDcholMixedCreate.argtypes = [C.POINTER(C.c_void_p), C.c_void_p, C.c_int, C.c_size_t, C.c_uint64,
                                         C.c_size_t, C.c_int, C.c_double, C.POINTER(C.c_long)]
        L.cuDcholMixedCreate.restype = C.c_int
        L.cuDcholMixedSolve.argtypes = [C.c_void_p, C.c_size_t, C.c_uint64, C.c_size_t, C.c_uint64, C.c_size_t,
                                        C.c_double, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.cuDcholMixedSolve.restype = C.c_int
        L.cuCholMixedGetFactor.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_size_t),
                                           C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.cuCholMixedDestroy.argtypes = [C.c_void_p]
        self.n = n
        self._p = C.c_void_p()
        info = C.c_long(0)
        rc = L.cuDcholMixedCreate(C.byref(self._p), h.value, _uplo(uplo), n, a, lda, precision, shift,
                                  C.byref(info))
        if rc != CUDA_SUCCESS:
            raise CuCholeskyError("cuDcholMixedCreate", rc)
        self.info = info.value

    def refactor(self) -> int:
        L = lib()
        L.cuDcholMixedRefactor.argtypes = [C.c_void_p, C.POINTER(C.c_long)]
        L.cuDcholMixedRefactor.restype = C.c_int
        info = C.c_long(0)
        rc = L.cuDcholMixedRefactor(self._p, C.byref(info))
        if rc != CUDA_SUCCESS:
            raise CuCholeskyError("cuDcholMixedRefactor", rc)
        self.info = info.value
        return self.info

    def solve(self, nrhs: int, b: int, ldb: int, x: int, ldx: int, tol: float = 0.0, maxit: int = 0):
        it = C.c_int(0)
        berr = C.c_double(0)
        rc = lib().cuDcholMixedSolve(self._p, nrhs, b, ldb, x, ldx, tol, maxit, C.byref(it), C.byref(berr))
        if rc != CUDA_SUCCESS:
            raise CuCholeskyError("cuDcholMixedSolve", rc)
        return it.value, berr.value

    def factor(self):
        """(W device pointer, ldw, s device pointer, |A|_inf, shift)."""
        w, s = C.c_uint64(0), C.c_uint64(0)
        ldw = C.c_size_t(0)
        anorm, shift = C.c_double(0), C.c_double(0)
        lib().cuCholMixedGetFactor(self._p, C.byref(w), C.byref(ldw), C.byref(s), C.byref(anorm), C.byref(shift))
        return w.value, ldw.value, s.value, anorm.value, shift.value

    def close(self):
        if self._p:
            lib().cuCholMixedDestroy(self._p)
            self._p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def call_syrk_lowp(h: Handle, precision: int, n: int, k: int, alpha: float, q: int, ldq: int, c: int,
                   ldc: int, stream: int = 0) -> int:
    """cuSsyrkLowp: C(lower) += alpha Q Q^T with BF16 / TF32 Q (k-major) and FP32 C."""
    L = lib()
    L.cuSsyrkLowp.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_size_t, C.c_float, C.c_uint64, C.c_size_t,
                              C.c_uint64, C.c_size_t, C.c_void_p]
    L.cuSsyrkLowp.restype = C.c_int
    return L.cuSsyrkLowp(h.value, precision, n, k, alpha, q, ldq, c, ldc, C.c_void_p(stream))


def call_posv_mixed(h: Handle, uplo: str, n: int, nrhs: int, a: int, lda: int, b: int, ldb: int, x: int,
                    ldx: int, precision: int = MIXED_TF32):
    """cuDposvMixed; returns (rc, iter, berr, info)."""
    L = lib()
    L.cuDposvMixed.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_size_t, C.c_uint64, C.c_size_t, C.c_uint64,
                               C.c_size_t, C.c_uint64, C.c_size_t, C.c_int, C.POINTER(C.c_int),
                               C.POINTER(C.c_double), C.POINTER(C.c_long)]
    L.cuDposvMixed.restype = C.c_int
    it, berr, info = C.c_int(0), C.c_double(0), C.c_long(0)
    rc = L.cuDposvMixed(h.value, _uplo(uplo), n, nrhs, a, lda, b, ldb, x, ldx, precision, C.byref(it),
                        C.byref(berr), C.byref(info))
    return rc, it.value, berr.value, info.value


# ---- host-memory routines (include/lapack.h cuMultiGPU*, include/cumultigpu.h) ----

def _declare_host(L: C.CDLL) -> None:
    if getattr(L, "_host_declared", False):
        return
    H = C.c_void_p
    L.cuMultiGPUCreate.argtypes = [C.POINTER(C.c_void_p), C.POINTER(C.c_int), C.c_int]
    L.cuMultiGPUDestroy.argtypes = [H]
    L.cuMultiGPUGetContextCount.argtypes = [H]
    L.cuMultiGPUSynchronize.argtypes = [H]
    L.cuMultiGPULAPACKCreate.argtypes = [C.POINTER(C.c_void_p), H]
    L.cuMultiGPULAPACKDestroy.argtypes = [H]
    L.cuMultiGPULAPACKSynchronize.argtypes = [H]
    L.cuMultiGPULAPACKGetStats.argtypes = [H] + [C.POINTER(C.c_ulonglong)] * 3
    for f in (L.cuMultiGPUCreate, L.cuMultiGPUDestroy, L.cuMultiGPUGetContextCount, L.cuMultiGPUSynchronize,
              L.cuMultiGPULAPACKCreate, L.cuMultiGPULAPACKDestroy, L.cuMultiGPULAPACKSynchronize,
              L.cuMultiGPULAPACKGetStats):
        f.restype = C.c_int
    for p in "SDCZ":
        for name in ("potrf", "lauum", "potri"):
            f = getattr(L, f"cuMultiGPU{p}{name}")
            f.argtypes = [H, C.c_int, C.c_size_t, C.c_void_p, C.c_size_t, C.POINTER(C.c_long)]
            f.restype = C.c_int
        f = getattr(L, f"cuMultiGPU{p}trtri")
        f.argtypes = [H, C.c_int, C.c_int, C.c_size_t, C.c_void_p, C.c_size_t, C.POINTER(C.c_long)]
        f.restype = C.c_int
    L._host_declared = True


class MultiGPU:
    """CUmultiGPU: the list of devices a host-memory handle may use."""

    def __init__(self, devices=(0,)):
        L = lib()
        _declare_host(L)
        self._m = C.c_void_p()
        arr = (C.c_int * len(devices))(*devices)
        rc = L.cuMultiGPUCreate(C.byref(self._m), arr, len(devices))
        if rc != CUDA_SUCCESS:
            raise CuCholeskyError("cuMultiGPUCreate", rc)

    @property
    def value(self) -> C.c_void_p:
        return self._m

    def count(self) -> int:
        return lib().cuMultiGPUGetContextCount(self._m)

    def synchronize(self) -> int:
        return lib().cuMultiGPUSynchronize(self._m)

    def close(self) -> None:
        if self._m:
            lib().cuMultiGPUDestroy(self._m)
            self._m = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HostHandle:
    """CUmultiGPULAPACKhandle over a MultiGPU (host-memory ?potrf/?trtri/?lauum/?potri)."""

    def __init__(self, mgpu: MultiGPU):
        L = lib()
        _declare_host(L)
        self._h = C.c_void_p()
        rc = L.cuMultiGPULAPACKCreate(C.byref(self._h), mgpu.value)
        if rc != CUDA_SUCCESS:
            raise CuCholeskyError("cuMultiGPULAPACKCreate", rc)

    @property
    def value(self) -> C.c_void_p:
        return self._h

    def synchronize(self) -> int:
        return lib().cuMultiGPULAPACKSynchronize(self._h)

    def stats(self) -> tuple[int, int, int]:
        """(kernels launched, bytes host->device, bytes device->host) since creation."""
        v = [C.c_ulonglong(0) for _ in range(3)]
        rc = lib().cuMultiGPULAPACKGetStats(self._h, *[C.byref(x) for x in v])
        if rc != CUDA_SUCCESS:
            raise CuCholeskyError("cuMultiGPULAPACKGetStats", rc)
        return tuple(x.value for x in v)

    def close(self) -> None:
        if self._h:
            lib().cuMultiGPULAPACKDestroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def call_host(hh, prefix: str, routine: str, uplo: str, n: int, ptr: int, lda: int,
              diag: str = "N") -> tuple[int, int]:
    """cuMultiGPU{prefix}{routine} on a column-major matrix at host address `ptr`
    (a numpy array's ``ctypes.data`` or a pinned torch tensor's ``data_ptr()``);
    returns (CUresult, info).  `hh` may be None to exercise the argument checks."""
    L = lib()
    _declare_host(L)
    info = C.c_long(0)
    f = getattr(L, f"cuMultiGPU{prefix}{routine}")
    h = hh.value if hh is not None else None
    if routine == "trtri":
        rc = f(h, _uplo(uplo), ord(diag.upper()), n, ptr, lda, C.byref(info))
    else:
        rc = f(h, _uplo(uplo), n, ptr, lda, C.byref(info))
    return rc, info.value


# ---- device RNG (include/curng.h) and the SPD generator cu?latmc -----------------

_RNG_FILL = {"raw": "Get", "oo": "GetOpenOpen", "oc": "GetOpenClose", "co": "GetCloseOpen", "cc": "GetCloseClose"}


class Rng:
    """CUrng32 (bits=32) or CUrng64 (bits=64) of the Philox4x32-10 type."""

    def __init__(self, bits: int = 64, seed: int | None = None):
        L = lib()
        self.bits = bits
        self._p = f"cuRng{bits}"
        self._g = C.c_void_p()
        typ = C.c_void_p.in_dll(L, "philox32_t" if bits == 32 else "philox64_t")
        f = getattr(L, self._p + "Create")
        f.argtypes = [C.POINTER(C.c_void_p), C.c_void_p]
        f.restype = C.c_int
        rc = f(C.byref(self._g), typ)
        if rc != CUDA_SUCCESS:
            raise CuCholeskyError(self._p + "Create", rc)
        if seed is not None:
            self.set(seed)

    @property
    def value(self) -> C.c_void_p:
        return self._g

    def set(self, seed: int) -> int:
        f = getattr(lib(), self._p + "Set")
        f.argtypes = [C.c_void_p, C.c_uint32 if self.bits == 32 else C.c_uint64]
        f.restype = C.c_int
        return f(self._g, seed)

    def fill(self, ptr: int, n: int, kind: str = "raw") -> int:
        """cuRng{32,64}{Get, GetOpenOpen, ...} into device memory at ptr (legacy stream)."""
        f = getattr(lib(), self._p + _RNG_FILL[kind])
        f.argtypes = [C.c_void_p, C.c_uint64, C.c_size_t]
        f.restype = C.c_int
        return f(self._g, ptr, n)

    def close(self) -> None:
        if self._g:
            f = getattr(lib(), self._p + "Destroy")
            f.argtypes = [C.c_void_p]
            f(self._g)
            self._g = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def call_latmc(prefix: str, rng, n: int, c: float, ptr: int, lda: int, stream: int = 0) -> int:
    """cu{S,D,C,Z}latmc: Hermitian positive definite n x n matrix with condition number
    c from the generator's stream (rng=None exercises the argument checks)."""
    f = getattr(lib(), f"cu{prefix}latmc")
    f.argtypes = [C.c_void_p, C.c_size_t, C.c_float if prefix in "SC" else C.c_double, C.c_uint64, C.c_size_t,
                  C.c_void_p]
    f.restype = C.c_int
    return f(rng.value if rng is not None else None, n, c, ptr, lda, C.c_void_p(stream))
