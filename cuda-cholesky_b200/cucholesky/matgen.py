"""Seeded synthetic SPD / HPD inputs with the shapes and value distributions of
the workloads this library is measured on.

Host generator: numpy's PCG64 (``np.random.default_rng(seed)``).  Device
generator (large n): torch's Philox on CUDA (``torch.Generator('cuda')``); the
matrix product that forms A is harness work done with torch, not the measured
path.

* ``spd_uniform``   A = G G^T / n + I, G i.i.d. uniform[-1, 1]   (real)
* ``hpd_normal``    A = G G^H / n + I, G complex normal, Re/Im ~ N(0, 1/2)
* ``sqexp_kernel``  K_ij = exp(-|x_i - x_j|^2 / (2 * 0.3^2)) + 1e-4 delta_ij,
                    x uniform in the unit cube (batched small matrices)
* ``scaled_spd``    A = D (G G^T / n + 1e-3 I) D, G i.i.d. N(0, 1),
                    D = diag(10^(k i / (n - 1))): kappa from ~1e3 (k = 0) to ~1e9
                    (k = 3), the mixed-precision solve's inputs; ``scaled_spd_device``
                    builds the same family on the GPU for large n
"""
from __future__ import annotations

import numpy as np

_REAL = {"s": np.float32, "d": np.float64, "c": np.float32, "z": np.float64}
_DT = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}


def dtype_of(p: str):
    return _DT[p]


def spd(p: str, n: int, seed: int = 0, lda: int | None = None) -> np.ndarray:
    """Column-major SPD (real p) or HPD (complex p) matrix of order n, computed in
    FP64 and rounded to the routine's type.  With lda > n the array has lda rows
    (the extra rows are padding, filled with a sentinel)."""
    rng = np.random.default_rng(seed)
    if p in "sd":
        G = rng.uniform(-1.0, 1.0, size=(n, n))
        A = G @ G.T / n + np.eye(n)
    else:
        G = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) * np.sqrt(0.5)
        A = G @ G.conj().T / n + np.eye(n)
        A[np.diag_indices(n)] = A[np.diag_indices(n)].real
    lda = n if lda is None else lda
    out = np.full((lda, n), 7.0, dtype=_DT[p], order="F")
    out[:n, :n] = A.astype(_DT[p])
    return out


def sqexp_kernel(n: int, rng: np.random.Generator, p: str = "d") -> np.ndarray:
    x = rng.uniform(0.0, 1.0, size=(n, 3))
    d2 = ((x[:, None, :] - x[None, :, :]) ** 2).sum(-1)
    K = np.exp(-d2 / (2 * 0.3 ** 2)) + 1e-4 * np.eye(n)
    return np.asfortranarray(K.astype(_DT[p]))


def backward_error(A: np.ndarray, F: np.ndarray, uplo: str) -> float:
    """||A - L L^H||_F / (n eps ||A||_F) for the factor stored in F's `uplo`
    triangle (A Hermitian, only its `uplo` triangle is trusted)."""
    n = A.shape[1]
    Af = _full_herm(A[:n, :n], uplo).astype(np.complex128 if np.iscomplexobj(A) else np.float64)
    if uplo == "L":
        L = np.tril(F[:n, :n]).astype(Af.dtype)
        R = L @ L.conj().T
    else:
        U = np.triu(F[:n, :n]).astype(Af.dtype)
        R = U.conj().T @ U
    eps = np.finfo(_REAL[_code(A)]).eps
    return float(np.linalg.norm(Af - R) / (n * eps * np.linalg.norm(Af)))


def inverse_residual(A: np.ndarray, Ainv: np.ndarray, uplo: str) -> float:
    """||I - A Ainv||_F / (n kappa eps) with kappa the 2-norm condition number."""
    n = A.shape[1]
    Af = _full_herm(A[:n, :n], uplo).astype(np.complex128 if np.iscomplexobj(A) else np.float64)
    Xf = _full_herm(Ainv[:n, :n], uplo).astype(Af.dtype)
    kappa = np.linalg.cond(Af)
    eps = np.finfo(_REAL[_code(A)]).eps
    return float(np.linalg.norm(np.eye(n) - Af @ Xf) / (n * kappa * eps))


def _code(A: np.ndarray) -> str:
    return {np.dtype(np.float32): "s", np.dtype(np.float64): "d",
            np.dtype(np.complex64): "c", np.dtype(np.complex128): "z"}[A.dtype]


def _full_herm(T: np.ndarray, uplo: str) -> np.ndarray:
    if uplo == "L":
        L = np.tril(T)
        F = L + np.tril(L, -1).conj().T
    else:
        U = np.triu(T)
        F = U + np.triu(U, 1).conj().T
    F = F.copy()
    F[np.diag_indices(F.shape[0])] = F[np.diag_indices(F.shape[0])].real
    return F


def scaled_spd(n: int, k: float, seed: int = 0) -> np.ndarray:
    """Column-major FP64 A = D (G G^T / n + 1e-3 I) D (see the module docstring)."""
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((n, n))
    d = 10.0 ** (k * np.arange(n) / max(n - 1, 1))
    A = (G @ G.T / n + 1e-3 * np.eye(n)) * d[:, None] * d[None, :]
    return np.asfortranarray(A)


def scaled_spd_device(n: int, k: float, seed: int = 0, device: str = "cuda"):
    """The ``scaled_spd`` family generated on the device (torch Philox normals,
    FP64 product with torch): returns a torch tensor T of shape (n, n) whose
    transpose is the column-major matrix (A is symmetric, so T itself is A)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    G = torch.randn((n, n), generator=g, device=device, dtype=torch.float64)
    A = G @ G.T
    A /= n
    A.diagonal().add_(1e-3)
    d = 10.0 ** (k * torch.arange(n, device=device, dtype=torch.float64) / max(n - 1, 1))
    A *= d[:, None]
    A *= d[None, :]
    del G
    return A
