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


# ---------------------------------------------------------------------------------
# Device-side inputs and error estimates for large orders (torch, FP64 arithmetic).
# A device matrix is a torch tensor T of shape (n, n) holding the column-major
# matrix M, i.e. M = T.T (T[j, i] = M(i, j)); for a Hermitian input T = conj(M).
# ---------------------------------------------------------------------------------
_TORCH_DT = {"s": "float32", "d": "float64", "c": "complex64", "z": "complex128"}
_EPS = {"s": 2.0 ** -23, "d": 2.0 ** -52, "c": 2.0 ** -23, "z": 2.0 ** -52}


def spd_device(p: str, n: int, seed: int = 0, device: str = "cuda"):
    """The ``spd`` family on the device (torch Philox, FP64 product), returned as
    the FP64 / complex128 tensor T of the column-major matrix (see above); round it
    to the routine's type with ``T.to(torch_dtype(p))``."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    if p in "sd":
        G = torch.rand((n, n), generator=g, device=device, dtype=torch.float64) * 2 - 1
        A = G @ G.T
    else:
        G = torch.randn((n, n), generator=g, device=device, dtype=torch.complex128)   # Re, Im ~ N(0, 1/2)
        A = G @ G.conj().T
    del G
    A /= n
    A.diagonal().add_(1.0)
    if p in "cz":
        A.diagonal().imag.zero_()
    return A.T.contiguous() if p in "cz" else A     # T = M^T (= conj(M) for Hermitian M)


def torch_dtype(p: str):
    import torch
    return getattr(torch, _TORCH_DT[p])


def _wide(T):
    import torch
    return T.to(torch.complex128 if T.is_complex() else torch.float64)


def factor_of(T, uplo: str):
    """L with A = L L^H from the factor a cu?potrf call left in T (FP64 copy)."""
    import torch
    M = _wide(T).T
    if uplo == "L":
        return torch.tril(M)
    return torch.triu(M).conj().T.contiguous()


def hermitian_of(T, uplo: str):
    """The full Hermitian matrix whose `uplo` triangle T holds (FP64 copy)."""
    import torch
    M = _wide(T).T
    H = torch.tril(M) if uplo == "L" else torch.triu(M)
    off = torch.tril(H, -1) if uplo == "L" else torch.triu(H, 1)
    H = H + off.conj().T
    if H.is_complex():
        H.diagonal().imag.zero_()
    return H


def _probes(n, k, like, seed):
    import torch
    g = torch.Generator(device=like.device)
    g.manual_seed(seed)
    return torch.randn((n, k), generator=g, device=like.device, dtype=like.dtype)


def probe_backward_error(A, L, p: str, k: int = 8, seed: int = 1234) -> float:
    """||A - L L^H||_F / (n eps ||A||_F) estimated with k Gaussian probes X:
    E[||E X||_F^2] = k ||E||_F^2.  A: full FP64 matrix, L: FP64 factor."""
    import torch
    n = A.shape[0]
    X = _probes(n, k, A, seed)
    R = A @ X - L @ (L.conj().T @ X)
    return float(torch.linalg.norm(R).item() / k ** 0.5 / (n * _EPS[p] * torch.linalg.norm(A).item()))


def cond2(A, Ainv, iters: int = 60, seed: int = 99) -> float:
    """2-norm condition number of Hermitian positive definite A from power
    iterations on A and on its computed inverse (a slight underestimate)."""
    import torch

    def lmax(M):
        v = _probes(M.shape[0], 1, M, seed)
        lam = 0.0
        for _ in range(iters):
            w = M @ v
            lam = torch.linalg.norm(w).item()
            v = w / lam
        return lam
    return lmax(A) * lmax(Ainv)


def probe_inverse_residual(A, Ainv, p: str, kappa: float | None = None, k: int = 8, seed: int = 4321) -> float:
    """||I - A Ainv||_F / (n kappa eps) estimated with k Gaussian probes."""
    import torch
    n = A.shape[0]
    if kappa is None:
        kappa = cond2(A, Ainv)
    X = _probes(n, k, A, seed)
    R = X - A @ (Ainv @ X)
    return float(torch.linalg.norm(R).item() / k ** 0.5 / (n * kappa * _EPS[p]))
