"""strttf / stfttr / rfp_diag_indices / add_to_diagonal on the GPU: bit-exact
against LAPACK golden vectors and the oracle (reference
python_tests/test_stfttr_strttf.py, python_tests/test_spftrs.py:133-166)."""
import numpy as np
import pytest
import torch

from conftest import VARIANTS
from helpers import TR, UL, dev, host

NS = [1, 2, 3, 4, 5, 6, 7, 8, 9, 15, 16, 17, 32, 33, 64, 65, 97]


@pytest.mark.gpu
@pytest.mark.parametrize("n", NS)
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_strttf_golden(curfp, golden, n, tr, ul):
    S = golden[f"S_{n}"].astype(np.float32)
    # only the stored triangle may be read: poison the other one with NaN
    Sp = S.copy()
    Sp[np.triu_indices(n, 1) if ul == 0 else np.tril_indices(n, -1)] = np.nan
    arf = curfp.strttf(dev(Sp), transr=TR[tr], uplo=UL[ul])
    assert np.array_equal(host(arf), golden[f"strttf_{n}_{TR[tr]}{UL[ul]}"].astype(np.float32))


@pytest.mark.gpu
@pytest.mark.parametrize("n", NS)
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_stfttr_golden(curfp, golden, n, tr, ul):
    arf = golden[f"strttf_{n}_{TR[tr]}{UL[ul]}"].astype(np.float32)
    A = host(curfp.stfttr(dev(arf), transr=TR[tr], uplo=UL[ul]))
    S = golden[f"S_{n}"].astype(np.float32)
    mask = np.triu(np.ones((n, n), bool)) if ul else np.tril(np.ones((n, n), bool))
    assert np.array_equal(A[mask], S[mask])
    assert not A[~mask].any()  # other triangle untouched (zero-initialised)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 5, 6, 33, 64, 97])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_raw_lda_and_untouched(curfp, orc, n, tr, ul):
    """lda > n; stfttr writes only the stored triangle of the destination."""
    lda = n + 3
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, lda)).astype(np.float32)
    arf = torch.empty(n * (n + 1) // 2, device="cuda")
    with curfp.Handle() as h:
        curfp.strttf_raw(h, tr, ul, n, dev(A), lda, arf)
        ref = orc.strttf(tr, ul, n, A.astype(np.float64), lda)
        assert np.array_equal(host(arf), ref.astype(np.float32))
        D = np.full((n, lda), 7.0, np.float32)
        Dd = dev(D)
        curfp.stfttr_raw(h, tr, ul, n, arf, Dd, lda)
    out = host(Dd)
    exp = orc.stfttr(tr, ul, n, ref, lda).astype(np.float32)
    mask = np.zeros((n, lda), bool)
    mask[:, :n] = np.triu(np.ones((n, n), bool)) if ul else np.tril(np.ones((n, n), bool))
    assert np.array_equal(out[mask], exp[mask])
    assert np.all(out[~mask] == 7.0)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [4095, 4096])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_round_trip_large(curfp, orc, n, tr, ul):
    """strttf -> stfttr round trip of triu/tril(N(0,1)) at n = 4095/4096,
    bit-exact, plus strttf against the oracle."""
    g = torch.Generator(device="cuda").manual_seed(n + tr * 2 + ul)
    M = torch.randn(n, n, device="cuda", generator=g)
    M = torch.triu(M) if ul else torch.tril(M)
    arf = curfp.strttf(M, transr=TR[tr], uplo=UL[ul])
    back = curfp.stfttr(arf, transr=TR[tr], uplo=UL[ul])
    assert torch.equal(back, M)
    arf2 = curfp.strttf(back, transr=TR[tr], uplo=UL[ul])
    assert torch.equal(arf2, arf)
    idx = curfp.rfp_diag_indices(n, transr=TR[tr], uplo=UL[ul])
    assert torch.equal(arf[idx], torch.diagonal(M))
    if n == 4095:
        ref = orc.strttf(tr, ul, n, host(M).astype(np.float64))
        assert np.array_equal(host(arf), ref.astype(np.float32))


@pytest.mark.gpu
@pytest.mark.parametrize("n", NS + [4095, 4096, 100001])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_diag_indices(curfp, orc, n, tr, ul):
    idx = host(curfp.rfp_diag_indices(n, transr=TR[tr], uplo=UL[ul]))
    assert idx.dtype == np.int64
    assert np.array_equal(idx, orc.diag_indices(tr, ul, n))


@pytest.mark.gpu
@pytest.mark.parametrize("n", NS)
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_diag_indices_golden(curfp, golden, n, tr, ul):
    idx = host(curfp.rfp_diag_indices(n, transr=TR[tr], uplo=UL[ul]))
    assert np.array_equal(idx, golden[f"diag_{n}_{TR[tr]}{UL[ul]}"])


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_add_to_diagonal(curfp, orc, dtype, tr, ul):
    n = 37
    C = torch.arange(n * (n + 1) // 2, dtype=dtype, device="cuda")
    exp = host(C).copy()
    exp[orc.diag_indices(tr, ul, n)] += 2.5
    curfp.add_to_diagonal(C, 2.5, transr=TR[tr], uplo=UL[ul])
    assert np.array_equal(host(C), exp)
