"""ssfrk / ssfr2k / spftrf / spftrs / spftri on the GPU against the LAPACK
golden vectors, the oracle and the reference's known-answer tests, all 8
variants (reference python_tests/test_vs_lapack.py, test_ssfrk.py,
test_spftrf.py, test_spftrs.py, test_spftri.py, test_ssfr2k.py).
Tolerances are those of the reference tests: max-abs 1e-3 on O(1) data for
the pipeline (test_vs_lapack.py:22-23) and 1e-4 on KATs."""
import numpy as np
import pytest
import torch

from conftest import VARIANTS
from helpers import TR, UL, dev, host

NS = [1, 2, 3, 4, 5, 6, 7, 8, 9, 15, 16, 17, 32, 33, 64, 65, 97]
TOL = 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("n", NS)
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_pipeline_vs_lapack(curfp, golden, n, tr, ul):
    kk = f"{n}_{TR[tr]}{UL[ul]}"
    k = max(1, n // 2)
    A = golden[f"A_{n}"].astype(np.float32)              # (n, k) row-major
    C = torch.empty(n * (n + 1) // 2, device="cuda")
    curfp.ssfrk(dev(A), C, transr=TR[tr], uplo=UL[ul])   # trans='T': A @ A.T
    np.testing.assert_allclose(host(C), golden[f"ssfrk_{kk}"], rtol=0, atol=TOL)
    curfp.add_to_diagonal(C, 1.0, transr=TR[tr], uplo=UL[ul])
    assert curfp.spftrf(C, transr=TR[tr], uplo=UL[ul]) == 0
    np.testing.assert_allclose(host(C), golden[f"spftrf_{kk}"], rtol=0, atol=TOL)
    B = dev(golden[f"B_{n}"].astype(np.float32))
    curfp.spftrs(C, B, transr=TR[tr], uplo=UL[ul])
    np.testing.assert_allclose(host(B), golden[f"spftrs_{kk}"], rtol=0, atol=TOL)
    Ci = C.clone()
    curfp.spftri(Ci, transr=TR[tr], uplo=UL[ul])
    np.testing.assert_allclose(host(Ci), golden[f"spftri_{kk}"], rtol=0, atol=TOL)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [63, 64, 65, 128, 129, 200, 257, 300])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_pipeline_vs_oracle(curfp, orc, n, tr, ul):
    """Sizes that exercise the recursive blocking (tiles of 64)."""
    rng = np.random.default_rng(n * 17 + tr * 2 + ul)
    k = max(1, n // 2)
    A = (rng.standard_normal((n, k)) / np.sqrt(k)).astype(np.float32)
    C = torch.empty(n * (n + 1) // 2, device="cuda")
    curfp.ssfrk(dev(A), C, transr=TR[tr], uplo=UL[ul])
    Co = orc.ssfrk(tr, ul, 1, n, k, 1.0, A.astype(np.float64), k, 0.0,
                   np.zeros(n * (n + 1) // 2))
    np.testing.assert_allclose(host(C), Co, rtol=0, atol=1e-5)
    curfp.add_to_diagonal(C, 1.0, transr=TR[tr], uplo=UL[ul])
    Co[orc.diag_indices(tr, ul, n)] += 1.0
    assert curfp.spftrf(C, transr=TR[tr], uplo=UL[ul]) == 0
    Fo, info = orc.spftrf(tr, ul, n, Co)
    np.testing.assert_allclose(host(C), Fo, rtol=0, atol=1e-4)
    B = rng.standard_normal((n, 5)).astype(np.float32)
    Bd = dev(B)
    curfp.spftrs(C, Bd, transr=TR[tr], uplo=UL[ul])
    Xo = orc.spftrs(tr, ul, n, 5, Fo, B.T.ravel(), n).reshape(5, n).T
    np.testing.assert_allclose(host(Bd), Xo, rtol=0, atol=1e-3)
    curfp.spftri(C, transr=TR[tr], uplo=UL[ul])
    Io, _ = orc.spftri(tr, ul, n, Fo)
    np.testing.assert_allclose(host(C), Io, rtol=0, atol=1e-3)


@pytest.mark.gpu
@pytest.mark.parametrize("tr,ul", VARIANTS)
@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-0.5, 1.5), (2.0, 1.0), (0.0, 3.0)])
@pytest.mark.parametrize("n,k", [(1, 3), (5, 4), (70, 33), (130, 129), (257, 64)])
def test_ssfrk_raw_vs_oracle(curfp, orc, tr, ul, trans, alpha, beta, n, k):
    rng = np.random.default_rng(n + k + trans)
    lda = n if trans == 0 else k
    # column-major op(A): trans=N -> A is n x k (storage k rows of n), trans=T -> k x n
    Araw = rng.standard_normal(lda * (k if trans == 0 else n)).astype(np.float32)
    C0 = rng.standard_normal(n * (n + 1) // 2).astype(np.float32)
    C = dev(C0)
    with curfp.Handle() as h:
        curfp.ssfrk_raw(h, tr, ul, trans, n, k, alpha, dev(Araw), lda, beta, C)
    exp = orc.ssfrk(tr, ul, trans, n, k, alpha, Araw, lda, beta, C0)
    np.testing.assert_allclose(host(C), exp, rtol=0, atol=2e-4 * max(1, k) ** 0.5)


@pytest.mark.gpu
@pytest.mark.parametrize("tr,ul", VARIANTS)
@pytest.mark.parametrize("n", [5, 6])
def test_ssfrk_quick_returns(curfp, tr, ul, n):
    """alpha=0,beta=1 pass-through; alpha=beta=0 zeroes C without reading A
    (A=NULL, reference tests/test_ssfrk.cu:38-66, test_ssfrk.py:12-56)."""
    nt = n * (n + 1) // 2
    C0 = torch.arange(1, nt + 1, dtype=torch.float32, device="cuda")
    C = C0.clone()
    with curfp.Handle() as h:
        curfp.ssfrk_raw(h, tr, ul, 1, n, 3, 0.0, None, 3, 1.0, C)
        torch.cuda.synchronize()
        assert torch.equal(C, C0)
        curfp.ssfrk_raw(h, tr, ul, 0, n, 1, 0.0, None, n, 0.0, C)
        torch.cuda.synchronize()
        assert not C.any()


@pytest.mark.gpu
def test_kats(curfp, golden):
    for name, n in [("kat_n2_NL", 2), ("kat_n3_NL", 3)]:
        A = dev(golden[f"{name}_in"].astype(np.float32))
        with curfp.Handle() as h:
            assert curfp.spftrf_raw(h, curfp.OP_N, curfp.FILL_LOWER, n, A) == 0
        np.testing.assert_allclose(host(A), golden[f"{name}_out"], atol=1e-4)
    C = dev(golden["kat_frk_n2_C"].astype(np.float32))
    A = dev(golden["kat_frk_n2_A"].astype(np.float32))
    with curfp.Handle() as h:
        curfp.ssfrk_raw(h, curfp.OP_N, curfp.FILL_LOWER, curfp.OP_N, 2, 1, 2.0, A, 2, 0.5, C)
    np.testing.assert_allclose(host(C), golden["kat_frk_n2_out"], atol=1e-4)
    for tr, ul in VARIANTS:
        x = torch.tensor([9.0], device="cuda")
        with curfp.Handle() as h:
            assert curfp.spftrf_raw(h, tr, ul, 1, x) == 0
        assert abs(x.item() - 3.0) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("tr,ul", VARIANTS)
@pytest.mark.parametrize("n,bad", [(6, 2), (6, 5), (7, 1), (7, 7), (150, 1), (150, 64),
                                   (150, 65), (150, 75), (150, 76), (150, 150)])
def test_spftrf_info(curfp, orc, tr, ul, n, bad):
    M = np.eye(n) * 2.0
    M[bad - 1, bad - 1] = -1.0
    C = dev(orc.strttf(tr, ul, n, M).astype(np.float32))
    info = curfp.spftrf(C, transr=TR[tr], uplo=UL[ul], check=False)
    assert info == bad
    with pytest.raises(torch.linalg.LinAlgError):
        curfp.spftrf(dev(orc.strttf(tr, ul, n, M).astype(np.float32)),
                     transr=TR[tr], uplo=UL[ul])


@pytest.mark.gpu
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_spftrf_nan_pivot(curfp, orc, tr, ul):
    n = 9
    M = np.eye(n)
    M[4, 4] = np.nan
    C = dev(orc.strttf(tr, ul, n, M).astype(np.float32))
    assert curfp.spftrf(C, transr=TR[tr], uplo=UL[ul], check=False) == 5


@pytest.mark.gpu
@pytest.mark.parametrize("tr,ul", VARIANTS)
@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("n,k", [(5, 3), (70, 20), (131, 65)])
def test_ssfr2k_vs_oracle(curfp, orc, tr, ul, trans, n, k):
    rng = np.random.default_rng(n * 3 + trans)
    lda = n if trans == 0 else k
    size = lda * (k if trans == 0 else n)
    A = rng.standard_normal(size).astype(np.float32)
    B = rng.standard_normal(size).astype(np.float32)
    C0 = rng.standard_normal(n * (n + 1) // 2).astype(np.float32)
    C = dev(C0)
    with curfp.Handle() as h:
        curfp.ssfr2k_raw(h, tr, ul, trans, n, k, 0.75, dev(A), lda, dev(B), lda, -0.5, C)
    exp = orc.ssfr2k(tr, ul, trans, n, k, 0.75, A, lda, B, lda, -0.5, C0)
    np.testing.assert_allclose(host(C), exp, rtol=0, atol=1e-4 * k)


@pytest.mark.gpu
def test_ssfr2k_high_level(curfp, orc):
    n, k = 40, 7
    rng = np.random.default_rng(5)
    A = rng.standard_normal((n, k)).astype(np.float32)
    B = rng.standard_normal((n, k)).astype(np.float32)
    C = torch.zeros(n * (n + 1) // 2, device="cuda")
    curfp.ssfr2k(dev(A), dev(B), C)   # trans='T': A, B row-major n x k
    exp = orc.ssfr2k(1, 1, 1, n, k, 1.0, A, k, B, k, 0.0, np.zeros(n * (n + 1) // 2))
    np.testing.assert_allclose(host(C), exp, rtol=0, atol=1e-4)


@pytest.mark.gpu
def test_errors(curfp):
    C = torch.zeros(10, device="cuda")
    with pytest.raises(ValueError):
        curfp.ssfrk(torch.zeros(4, 2, device="cuda", dtype=torch.float64), C)
    with pytest.raises(ValueError):
        curfp.spftrf(torch.zeros(11, device="cuda"))
    with pytest.raises(ValueError):
        curfp.spftrs(C, torch.zeros(3, 2, device="cuda"))
    with pytest.raises(curfp.CurfpError, match="status=3"):
        with curfp.Handle() as h:
            curfp.ssfrk_raw(h, 0, 0, 0, -1, 2, 1.0, C, 4, 0.0, C)
    with pytest.raises(curfp.CurfpError, match="status=3"):
        with curfp.Handle() as h:
            curfp.strttf_raw(h, 0, 0, 4, torch.zeros(16, device="cuda"), 3, C)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 3])
def test_spftri_small_kats(curfp, orc, n):
    """spftri on hand-sized matrices, all variants (n=1 is 1/x^2)."""
    M = np.array([[4.0, 1, 0.5], [1, 3, 0.2], [0.5, 0.2, 2]])[:n, :n]
    for tr, ul in VARIANTS:
        C = dev(orc.strttf(tr, ul, n, M).astype(np.float32))
        curfp.spftrf(C, transr=TR[tr], uplo=UL[ul])
        curfp.spftri(C, transr=TR[tr], uplo=UL[ul])
        inv = orc.rfp_to_dense_sym(tr, ul, n, host(C).astype(np.float64))
        np.testing.assert_allclose(inv, np.linalg.inv(M), atol=1e-5)


@pytest.mark.gpu
def test_spftri_zero_pivot_fails(curfp, orc):
    n = 6
    M = np.eye(n)
    M[3, 3] = 0.0
    C = dev(orc.strttf(1, 1, n, M).astype(np.float32))
    before = C.clone()
    with pytest.raises(curfp.CurfpError, match="status=4"):
        curfp.spftri(C)
    assert torch.equal(C, before)


@pytest.mark.gpu
def test_streams(curfp, orc):
    """All routines on a non-default stream, with the tensors produced and
    consumed on that stream too (reference test_spftrs.py:169-188)."""
    n, k = 300, 40
    s = torch.cuda.Stream()
    rng = np.random.default_rng(1)
    A = (rng.standard_normal((n, k)) / np.sqrt(k)).astype(np.float32)
    B = rng.standard_normal((n, 3)).astype(np.float32)
    curfp.set_stream(s)
    try:
        with torch.cuda.stream(s):
            Ad, Bd = dev(A), dev(B)
            C = torch.empty(n * (n + 1) // 2, device="cuda")
            curfp.ssfrk(Ad, C)
            curfp.add_to_diagonal(C, 1.0)
            curfp.spftrf(C)
            curfp.spftrs(C, Bd)
            out = Bd.cpu()
    finally:
        s.synchronize()
        curfp.set_stream(None)
    Co = orc.ssfrk(1, 1, 1, n, k, 1.0, A, k, 0.0, np.zeros(n * (n + 1) // 2))
    Co[orc.diag_indices(1, 1, n)] += 1.0
    Fo, _ = orc.spftrf(1, 1, n, Co)
    Xo = orc.spftrs(1, 1, n, 3, Fo, B.T.ravel(), n).reshape(3, n).T
    np.testing.assert_allclose(out.numpy(), Xo, atol=1e-3)
