"""The batched plan (cu?cholBatchedCreate/Run/Results) through the C ABI: factor,
log det and inverse of many SPD matrices of uneven sizes in one graph launch,
against the oracle, with per-matrix info on a failing matrix."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import cucholesky as cc
from cucholesky import matgen

pytestmark = pytest.mark.gpu

EPS = {"d": np.finfo(np.float64).eps, "s": np.finfo(np.float32).eps}
NP = {"d": np.float64, "s": np.float32}


def _batch(p, sizes, seed):
    rng = np.random.default_rng(seed)
    mats = []
    for i, n in enumerate(sizes):
        if i % 2:
            mats.append(matgen.sqexp_kernel(n, rng, p))
        else:
            mats.append(matgen.spd(p, n, seed=seed + i))
    return mats


def _run(handle, p, mats, uplo, nb, flags=7, bad=None):
    import torch
    packed, off, sizes = cc.pack_colmajor(mats, NP[p])
    T = torch.from_numpy(packed).cuda()
    plan = cc.BatchedPlan(handle, T, sizes, off, uplo=uplo, flags=flags, nb=nb)
    plan.run()
    info, ld = plan.results()
    out = T.cpu().numpy()
    res = [np.asfortranarray(out[o:o + n * n].reshape(n, n, order="F")) for o, n in zip(off, sizes)]
    return plan, T, info, ld, res


# nb: 0 = the plan's tuner picks; 32 / 64 = the graph of grouped launches with that
# block size; -1 = the persistent kernel (FP64: one launch, matrices from a queue)
@pytest.mark.parametrize("p,nb", [("d", 0), ("d", 32), ("d", 64), ("d", -1), ("s", 0), ("s", 32), ("s", 64)])
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_batched_factor_logdet_inverse(handle, p, uplo, nb):
    sizes = [1, 7, 8, 31, 33, 64, 65, 100, 128, 129, 200, 257, 300, 17, 90, 512, 449]
    mats = _batch(p, sizes, seed=11)
    plan, T, info, ld, res = _run(handle, p, mats, uplo, nb)
    assert plan.nb in ((32, 64, -1) if p == "d" else (32, 64)) and (nb == 0 or plan.nb == nb)
    tri = np.tril if uplo == "L" else np.triu
    for A, inv, inf, l in zip(mats, res, info, ld):
        n = A.shape[0]
        F = A.copy(order="F")
        assert inf == O.potrf(p, uplo, F) == 0
        ref_ld = 2.0 * float(np.sum(np.log(np.diag(F).astype(np.float64))))
        assert abs(l - ref_ld) <= 100 * n * EPS[p] * max(1.0, abs(ref_ld)), (n, l, ref_ld)
        X = F.copy(order="F")
        assert O.potri(p, uplo, X) == 0
        scale = np.abs(X).max()
        d = np.abs(tri(inv) - tri(X)).max() / scale
        kappa = np.linalg.cond(A.astype(np.float64))
        assert d <= 50 * n * kappa * EPS[p], (n, d)
        if p == "d":
            assert matgen.inverse_residual(A, inv, uplo) <= 10, n


@pytest.mark.parametrize("nb", [64, -1])
def test_batched_failure_is_per_matrix(handle, nb):
    sizes = [50, 120, 200, 70]
    mats = _batch("d", sizes, seed=3)
    mats[2][150, 150] = -1.0            # matrix 2 fails at leading minor 151
    plan, T, info, ld, res = _run(handle, "d", mats, "L", nb)
    assert info == [0, 0, 151, 0]
    for b in (0, 1, 3):
        assert matgen.inverse_residual(mats[b], res[b], "L") <= 10
    # the plan runs again on refilled buffers with the same results
    import torch
    packed, off, _ = cc.pack_colmajor(mats, np.float64)
    T.copy_(torch.from_numpy(packed))
    plan.run()
    info2, ld2 = plan.results()
    assert info2 == info and np.allclose(ld2, ld)


@pytest.mark.parametrize("nb", [32, -1])
def test_batched_factor_only(handle, nb):
    sizes = [40, 80, 160]
    mats = _batch("d", sizes, seed=5)
    plan, T, info, ld, res = _run(handle, "d", mats, "L", nb, flags=cc.BATCHED_POTRF | cc.BATCHED_LOGDET)
    for A, F, inf in zip(mats, res, info):
        assert inf == 0
        assert matgen.backward_error(A, F, "L") <= 10
