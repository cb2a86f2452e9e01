"""FP64 (D-prefix) twins on the GPU against the FP64 oracle (the reference's
algorithm restated in C, pinned to LAPACK) and LAPACK, all 8 variants.

Bounds (FP64 summation-order spread): packing bit-exact; ssfrk / ssfr2k
1e-13 of the product scale; factor, solution and inverse 1e-11 relative on
O(1), well-conditioned data (cond ~ 10); norms 1e-12; the condition estimate
within 1e-9 of the oracle estimator on the same factor and within 3x of
LAPACK dpocon; symmetric multiplies and rank updates 1e-13."""
import numpy as np
import pytest
import scipy.linalg
import torch
from scipy.linalg import lapack

from conftest import VARIANTS
from helpers import TR, UL, host
from oracle import condest

NS = [1, 2, 3, 17, 64, 65, 200, 257]


def d64(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def spd_rfp(orc, tr, ul, n, seed, shift=1.0):
    rng = np.random.default_rng(seed)
    k = max(1, n // 2)
    A = rng.standard_normal((n, k)) / np.sqrt(k)
    C = orc.ssfrk(tr, ul, 1, n, k, 1.0, A, k, 0.0, np.zeros(n * (n + 1) // 2))
    C[orc.diag_indices(tr, ul, n)] += shift
    return A, C


@pytest.mark.gpu
@pytest.mark.parametrize("n", NS)
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_dpack_bit_exact(curfp, orc, n, tr, ul):
    M = np.random.default_rng(n).standard_normal((n, n))
    want = orc.strttf(tr, ul, n, M)
    arf = curfp.dstrttf(d64(M), transr=TR[tr], uplo=UL[ul])
    np.testing.assert_array_equal(host(arf), want)
    D = curfp.dstfttr(d64(want), transr=TR[tr], uplo=UL[ul])
    np.testing.assert_array_equal(host(D), orc.stfttr(tr, ul, n, want))


@pytest.mark.gpu
@pytest.mark.parametrize("n", NS)
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_dsfrk_dsfr2k(curfp, orc, n, tr, ul):
    rng = np.random.default_rng(3 * n + 1)
    k = max(1, n // 3)
    A, B = rng.standard_normal((n, k)), rng.standard_normal((n, k))
    C0 = rng.standard_normal(n * (n + 1) // 2)
    C = d64(C0)
    curfp.dsfrk(d64(A), C, alpha=0.5, beta=-2.0, transr=TR[tr], uplo=UL[ul])
    want = orc.ssfrk(tr, ul, 1, n, k, 0.5, A, k, -2.0, C0)
    assert np.abs(host(C) - want).max() <= 1e-13 * max(1.0, np.abs(want).max()) * k
    C = d64(C0)
    curfp.dsfr2k(d64(A), d64(B), C, alpha=0.25, beta=1.0, transr=TR[tr], uplo=UL[ul])
    want = orc.ssfr2k(tr, ul, 1, n, k, 0.25, A, k, B, k, 1.0, C0)
    assert np.abs(host(C) - want).max() <= 1e-13 * max(1.0, np.abs(want).max()) * k


@pytest.mark.gpu
@pytest.mark.parametrize("n", NS + [600, 1001])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_dpftrf_dpftrs_dpftri(curfp, orc, n, tr, ul):
    _, C = spd_rfp(orc, tr, ul, n, seed=n + 10 * tr + ul)
    F_want, info = orc.spftrf(tr, ul, n, C)
    assert info == 0
    F = d64(C)
    assert curfp.dpftrf(F, transr=TR[tr], uplo=UL[ul]) == 0
    np.testing.assert_allclose(host(F), F_want, rtol=1e-11, atol=1e-12)
    rng = np.random.default_rng(n)
    B = rng.standard_normal((7, n))  # column-major n x 7
    X = d64(B)
    curfp.dpftrs_raw(curfp._get_handle(), tr, ul, n, 7, F, X, n)
    X_want = orc.spftrs(tr, ul, n, 7, F_want, B.ravel(), n).reshape(7, n)
    np.testing.assert_allclose(host(X), X_want, rtol=1e-10, atol=1e-11)
    Z = F.clone()
    curfp.dpftri(Z, transr=TR[tr], uplo=UL[ul])
    Z_want, rc = orc.spftri(tr, ul, n, F_want)
    assert rc == 0
    np.testing.assert_allclose(host(Z), Z_want, rtol=1e-10, atol=1e-11)


@pytest.mark.gpu
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_dpftrf_info(curfp, orc, tr, ul):
    n, bad = 300, 170
    M = np.eye(n) * 2.0
    M[bad - 1, bad - 1] = -1.0
    arf = d64(orc.strttf(tr, ul, n, M))
    assert curfp.dpftrf(arf, transr=TR[tr], uplo=UL[ul], check=False) == bad
    with pytest.raises(torch.linalg.LinAlgError):
        curfp.dpftrf(d64(orc.strttf(tr, ul, n, M)), transr=TR[tr], uplo=UL[ul])


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 5, 64, 65, 300])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_dlansf_dpfcon(curfp, orc, n, tr, ul):
    _, C = spd_rfp(orc, tr, ul, n, seed=7 * n + tr + 2 * ul, shift=0.1)
    S = orc.rfp_to_dense_sym(tr, ul, n, C)
    arf = d64(C)
    kw = dict(transr=TR[tr], uplo=UL[ul])
    assert curfp.dlansf(arf, "M", **kw) == np.abs(S).max()
    one = np.abs(S).sum(axis=0).max()
    assert abs(curfp.dlansf(arf, "1", **kw) - one) <= 1e-12 * one
    fro = np.linalg.norm(S)
    assert abs(curfp.dlansf(arf, "F", **kw) - fro) <= 1e-12 * fro
    rcond = curfp.dpftrf_rcond(arf, **kw)
    L = orc.rfp_to_factor(tr, ul, n, host(arf))
    port = condest.spfcon(condest.dense_factor_solver(L), n, one)
    assert abs(rcond - port) <= 1e-9 * port, (rcond, port)
    want, info = lapack.dpocon(scipy.linalg.cholesky(S, lower=False), one)
    assert info == 0 and 1 / 3 <= rcond / want <= 3


@pytest.mark.gpu
@pytest.mark.parametrize("n,m", [(1, 3), (65, 7), (300, 40)])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_dsymm_and_rank_updates(curfp, orc, n, m, tr, ul):
    rng = np.random.default_rng(n + m)
    nt = n * (n + 1) // 2
    arf = rng.standard_normal(nt)
    S = orc.rfp_to_dense_sym(tr, ul, n, arf)
    B = rng.standard_normal((m, n))  # column-major n x m
    C0 = rng.standard_normal((m, n))
    Ct = d64(C0)
    curfp.dsfmm_raw(curfp._get_handle(), tr, ul, 0, n, m, 0.5, d64(arf), d64(B), n, 2.0, Ct, n)
    want = (0.5 * S @ B.T + 2.0 * C0.T).T
    assert np.abs(host(Ct) - want).max() <= 1e-13 * np.abs(want).max() * np.sqrt(n)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    yd = d64(y)
    curfp.dsfmv(d64(arf), d64(x), yd, alpha=1.5, beta=-1.0, transr=TR[tr], uplo=UL[ul])
    want = 1.5 * S @ x - y
    assert np.abs(host(yd) - want).max() <= 1e-13 * np.abs(want).max() * np.sqrt(n)
    a1 = d64(arf)
    curfp.dsfr(a1, d64(x), alpha=0.75, transr=TR[tr], uplo=UL[ul])
    got = orc.rfp_to_dense_sym(tr, ul, n, host(a1))
    np.testing.assert_allclose(got, S + 0.75 * np.outer(x, x), rtol=0, atol=1e-14 * 20)
    a2 = d64(arf)
    curfp.dsfr2(a2, d64(x), d64(y), alpha=-0.5, transr=TR[tr], uplo=UL[ul])
    got = orc.rfp_to_dense_sym(tr, ul, n, host(a2))
    np.testing.assert_allclose(got, S - 0.5 * (np.outer(x, y) + np.outer(y, x)), rtol=0,
                               atol=1e-14 * 40)


@pytest.mark.gpu
@pytest.mark.parametrize("tr,ul", [(1, 1), (0, 0)])
def test_dpftrf_large_backward_error(curfp, tr, ul):
    """n = 4097 through the recursive blocked path (SIMT DFMA GEMMs, the
    FP64 wavefront solve): ||C - L L^T||_F / ||C||_F and the solve's
    normwise backward error at FP64 level."""
    n, k = 4097, 512
    g = torch.Generator(device="cuda").manual_seed(9)
    A = torch.randn(n, k, device="cuda", dtype=torch.float64, generator=g) / k ** 0.5
    C = torch.empty(n * (n + 1) // 2, device="cuda", dtype=torch.float64)
    curfp.dsfrk(A, C, transr=TR[tr], uplo=UL[ul])
    curfp.add_to_diagonal(C, 1.0, transr=TR[tr], uplo=UL[ul])
    S = curfp.dstfttr(C, transr=TR[tr], uplo=UL[ul])
    S = S + (S.triu(1).T if ul else S.tril(-1).T)
    F = C.clone()
    assert curfp.dpftrf(F, transr=TR[tr], uplo=UL[ul]) == 0
    T = curfp.dstfttr(F, transr=TR[tr], uplo=UL[ul])
    L = T.T if ul else T
    assert (torch.linalg.norm(S - L @ L.T) / torch.linalg.norm(S)).item() <= 1e-14
    B = torch.randn(n, 16, device="cuda", dtype=torch.float64, generator=g)
    X = B.clone()
    curfp.dpftrs(F, X, transr=TR[tr], uplo=UL[ul])
    r = (B - S @ X).norm(dim=0) / (torch.linalg.norm(S) * X.norm(dim=0) + B.norm(dim=0))
    assert r.max().item() <= 1e-15
