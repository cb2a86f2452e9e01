"""Solves with few right-hand sides (nrhs <= 8) at sizes whose RFP rectangle
update (n/2 x n/2 >= 2^20 elements) goes through the bandwidth-bound
few-column kernels, all 8 variants, for every column-count instantiation
(1, 2, 3-4, 5-8) and 9 right-hand sides (the tiled kernel) beside them.

spftrs / dpftrs against an FP64 solve with the same factor (the GPU factor,
unpacked by the oracle, two dense triangular solves): max-abs error within
2e-5 (FP32) / 1e-12 (FP64) of max |X| -- the matrices are C = A A^T + I with
A ~ N(0, 1/64), cond(C) < 100.  Two runs on the same input agree bit for
bit (fixed summation order), and the few-column path reads the right-hand
sides through a leading dimension larger than n."""
import numpy as np
import pytest
import scipy.linalg
import torch

from conftest import VARIANTS
from helpers import TR, UL, host

NS = [2048, 2049, 4097]
NRHS = [1, 2, 3, 5, 8, 9]


def factor(curfp, n, tr, ul, dtype, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    A = torch.randn(n, 64, device="cuda", dtype=dtype, generator=g) / 8.0
    C = torch.empty(n * (n + 1) // 2, device="cuda", dtype=dtype)
    kw = dict(transr=TR[tr], uplo=UL[ul])
    if dtype == torch.float64:
        curfp.dsfrk(A, C, **kw)
        curfp.add_to_diagonal(C, 1.0, **kw)
        assert curfp.dpftrf(C, **kw) == 0
    else:
        curfp.ssfrk(A, C, **kw)
        curfp.add_to_diagonal(C, 1.0, **kw)
        assert curfp.spftrf(C, **kw) == 0
    return C


def fp64_solve(orc, tr, ul, n, F, B):
    L = orc.rfp_to_factor(tr, ul, n, host(F).astype(np.float64))
    Y = scipy.linalg.solve_triangular(L, B, lower=True)
    return scipy.linalg.solve_triangular(L, Y, lower=True, trans="T")


@pytest.mark.gpu
@pytest.mark.parametrize("n", NS)
@pytest.mark.parametrize("nrhs", NRHS)
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_spftrs_few_rhs(curfp, orc, n, nrhs, tr, ul):
    F = factor(curfp, n, tr, ul, torch.float32, seed=n + 7 * nrhs + 31 * tr + 63 * ul)
    rng = np.random.default_rng(n + nrhs)
    ldb = n + 3
    Bh = rng.standard_normal((nrhs, ldb)).astype(np.float32)  # column-major n x nrhs, ldb
    want = fp64_solve(orc, tr, ul, n, F, Bh[:, :n].T.astype(np.float64))
    h = curfp._get_handle()
    X1 = torch.from_numpy(Bh).cuda()
    X2 = X1.clone()
    curfp.spftrs_raw(h, tr, ul, n, nrhs, F, X1, ldb)
    curfp.spftrs_raw(h, tr, ul, n, nrhs, F, X2, ldb)
    assert torch.equal(X1, X2)
    got = host(X1)[:, :n].T.astype(np.float64)
    assert np.abs(got - want).max() <= 2e-5 * np.abs(want).max()
    np.testing.assert_array_equal(host(X1)[:, n:], Bh[:, n:])  # padding rows untouched


@pytest.mark.gpu
@pytest.mark.parametrize("nrhs", [1, 2, 4, 6, 9])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_dpftrs_few_rhs(curfp, orc, nrhs, tr, ul):
    n = 2049
    F = factor(curfp, n, tr, ul, torch.float64, seed=3 * nrhs + tr + 2 * ul)
    rng = np.random.default_rng(nrhs)
    B = rng.standard_normal((nrhs, n))
    want = fp64_solve(orc, tr, ul, n, F, B.T)
    X = torch.from_numpy(B.copy()).cuda()
    curfp.dpftrs_raw(curfp._get_handle(), tr, ul, n, nrhs, F, X, n)
    got = host(X).T
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [300, 513, 1000])
@pytest.mark.parametrize("nrhs", [2048, 2100])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_spftrs_many_rhs(curfp, orc, n, nrhs, tr, ul):
    """Thousands of right-hand sides over triangles of at most 512 rows (the
    recursive solve's leaves): one CTA per 64-column chunk walks the block
    rows (a partial last chunk with 2100 columns); against the FP64 solve
    with the same factor, and bitwise repeatable."""
    F = factor(curfp, n, tr, ul, torch.float32, seed=n + nrhs + 5 * tr + 11 * ul)
    rng = np.random.default_rng(n * nrhs)
    Bh = rng.standard_normal((nrhs, n)).astype(np.float32)  # column-major n x nrhs
    want = fp64_solve(orc, tr, ul, n, F, Bh.T.astype(np.float64))
    h = curfp._get_handle()
    X1 = torch.from_numpy(Bh).cuda()
    X2 = X1.clone()
    curfp.spftrs_raw(h, tr, ul, n, nrhs, F, X1, n)
    curfp.spftrs_raw(h, tr, ul, n, nrhs, F, X2, n)
    assert torch.equal(X1, X2)
    got = host(X1).T.astype(np.float64)
    assert np.abs(got - want).max() <= 2e-5 * np.abs(want).max()
