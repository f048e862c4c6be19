"""ctypes front end to the oracle libraries.  TEST INFRASTRUCTURE ONLY.

Two CPU implementations of the reference's dense SPD path sit behind the same
Python calls:

* ``impl="port"``      -> ``oracle/liboracle.so``, the plain-C restatement in
  ``oracle/oracle.c`` (always present after ``make -f oracle/Makefile``).
* ``impl="reference"`` -> ``oracle/_ref/libref.so``, the reference's own
  ``lapack/*.c`` over ``blas/*.c`` compiled from its sources by ``oracle/ref.mk``.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may import this module.  Matrices are numpy arrays in column-major
(Fortran) order; the routines work in place like the reference's, and return
``info`` with the reference's meaning (``lapack/dpotrf.c:86-114``).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref.so")

_DT = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}
_libs: dict[str, C.CDLL] = {}


def available(impl: str) -> bool:
    return os.path.exists(PORT_LIB if impl == "port" else REF_LIB)


def _lib(impl: str) -> C.CDLL:
    if impl not in _libs:
        path = PORT_LIB if impl == "port" else REF_LIB
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -f oracle/Makefile [ref REF=<reference tree>])")
        lib = C.CDLL(path)
        if impl == "reference":
            # the reference prints a message through its XERBLA hook on argument
            # errors (blas/xerbla.c:5-9); leave it installed
            pass
        _libs[impl] = lib
    return _libs[impl]


def _fn(impl: str, p: str, name: str):
    lib = _lib(impl)
    return getattr(lib, (f"orc_{p}{name}" if impl == "port" else f"{p}{name}"))


def _check(A: np.ndarray, p: str):
    if A.dtype != _DT[p]:
        raise TypeError(f"{p}-routines want {_DT[p]}, got {A.dtype}")
    if not A.flags.f_contiguous:
        raise ValueError("matrix must be column-major (Fortran order)")


def _uplo(impl: str, u: str):
    # the port takes a char, the reference a CBlasUplo enum whose values are the
    # same characters (include/blas.h:25)
    return C.c_char(u.encode()) if impl == "port" else C.c_int(ord(u))


def potrf(p: str, uplo: str, A: np.ndarray, lda: int | None = None, impl: str = "port") -> int:
    """In-place Cholesky factor of the `uplo` triangle; returns info."""
    _check(A, p)
    n = A.shape[1]
    lda = A.shape[0] if lda is None else lda
    info = C.c_long(0)
    _fn(impl, p, "potrf")(_uplo(impl, uplo), C.c_size_t(n), A.ctypes.data_as(C.c_void_p),
                          C.c_size_t(lda), C.byref(info))
    return info.value


def potri(p: str, uplo: str, A: np.ndarray, impl: str = "port") -> int:
    _check(A, p)
    info = C.c_long(0)
    _fn(impl, p, "potri")(_uplo(impl, uplo), C.c_size_t(A.shape[1]), A.ctypes.data_as(C.c_void_p),
                          C.c_size_t(A.shape[0]), C.byref(info))
    return info.value


def trtri(p: str, uplo: str, A: np.ndarray, diag: str = "N", impl: str = "port") -> int:
    _check(A, p)
    info = C.c_long(0)
    _fn(impl, p, "trtri")(_uplo(impl, uplo), _uplo(impl, diag), C.c_size_t(A.shape[1]),
                          A.ctypes.data_as(C.c_void_p), C.c_size_t(A.shape[0]), C.byref(info))
    return info.value


def lauum(p: str, uplo: str, A: np.ndarray, impl: str = "port") -> int:
    _check(A, p)
    info = C.c_long(0)
    _fn(impl, p, "lauum")(_uplo(impl, uplo), C.c_size_t(A.shape[1]), A.ctypes.data_as(C.c_void_p),
                          C.c_size_t(A.shape[0]), C.byref(info))
    return info.value


def logdet(p: str, x: np.ndarray, incx: int, n: int, impl: str = "port") -> float:
    """2 * sum(log(Re x[i*incx])) over a flat buffer `x`."""
    f = _fn(impl, p, "logdet")
    if impl == "port" or p in "dz":
        f.restype = C.c_double
    else:
        f.restype = C.c_float
    return float(f(x.ctypes.data_as(C.c_void_p), C.c_size_t(incx), C.c_size_t(n)))


def set_threads(n: int) -> None:
    """OpenMP thread count for both libraries (they share libgomp)."""
    try:
        gomp = C.CDLL("libgomp.so.1")
        gomp.omp_set_num_threads(C.c_int(int(n)))
    except OSError:
        os.environ["OMP_NUM_THREADS"] = str(n)
