"""Parity with the reference's own GPU build (oracle/_ref/libcurfp_ref.so,
the unmodified reference sources on cuBLAS/cuSOLVER) on the same inputs.

Bit-exact for strttf/stfttr/diag; for the floating-point routines the bounds
are stated per quantity on O(1) data (cond ~ 45): ssfrk max-abs 1e-5, factor
max-abs 1e-4, solution and inverse max-relative 1e-4 / 2e-4 -- the spread of
two FP32 summation orders of the same algorithm (both results are compared
with FP64 elsewhere)."""
import numpy as np
import pytest
import torch

from conftest import VARIANTS
from helpers import REF_LIB, TR, UL, RefLib, dev, host

pytestmark = pytest.mark.skipif(not REF_LIB.exists(),
                                reason="reference build missing (make -C oracle ref)")


@pytest.fixture(scope="module")
def ref():
    return RefLib()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 3, 64, 65, 255, 256, 1023])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_pack_bit_exact_vs_reference(curfp, ref, n, tr, ul):
    g = torch.Generator(device="cuda").manual_seed(n)
    M = torch.randn(n, n, device="cuda", generator=g)
    a_ref = torch.empty(n * (n + 1) // 2, device="cuda")
    assert ref.strttf(tr, ul, n, M, n, a_ref) == 0
    a_our = curfp.strttf(M, transr=TR[tr], uplo=UL[ul])
    torch.cuda.synchronize()
    assert torch.equal(a_our, a_ref)
    D_ref = torch.zeros(n, n, device="cuda")
    assert ref.stfttr(tr, ul, n, a_ref, D_ref, n) == 0
    D_our = curfp.stfttr(a_ref, transr=TR[tr], uplo=UL[ul])
    torch.cuda.synchronize()
    assert torch.equal(D_our, D_ref)


@pytest.mark.gpu
@pytest.mark.parametrize("n,k", [(64, 32), (65, 32), (1000, 128), (1001, 128)])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_pipeline_vs_reference(curfp, ref, orc, n, k, tr, ul):
    g = torch.Generator(device="cuda").manual_seed(n + 10 * tr + ul)
    A = torch.randn(n, k, device="cuda", generator=g) / k ** 0.5
    nt = n * (n + 1) // 2
    C_ref = torch.empty(nt, device="cuda")
    C_our = torch.empty(nt, device="cuda")
    assert ref.ssfrk(tr, ul, 1, n, k, 1.0, A, k, 0.0, C_ref) == 0
    curfp.ssfrk(A, C_our, transr=TR[tr], uplo=UL[ul])
    torch.cuda.synchronize()
    d = (C_our - C_ref).abs().max().item()
    assert d <= 1e-5, d
    curfp.add_to_diagonal(C_ref, 1.0, transr=TR[tr], uplo=UL[ul])
    C_our.copy_(C_ref)
    A0 = host(C_ref).astype(np.float64)
    st, info = ref.spftrf(tr, ul, n, C_ref)
    assert st == 0 and info == 0
    assert curfp.spftrf(C_our, transr=TR[tr], uplo=UL[ul]) == 0
    # factors agree to FP32 rounding (cond(A) ~ 45 here)
    d = (C_our - C_ref).abs().max().item()
    assert d <= 1e-4, d
    B = torch.randn(64, n, device="cuda", generator=g)  # column-major n x 64
    X_ref, X_our = B.clone(), B.clone()
    assert ref.spftrs(tr, ul, n, 64, C_ref, X_ref, n) == 0
    with curfp.Handle() as h:
        curfp.spftrs_raw(h, tr, ul, n, 64, C_our, X_our, n)
    torch.cuda.synchronize()
    rel = ((X_our - X_ref).abs().max() / X_ref.abs().max()).item()
    assert rel <= 1e-4, rel
    I_ref, I_our = C_ref.clone(), C_our.clone()
    assert ref.spftri(tr, ul, n, I_ref) == 0
    curfp.spftri(I_our, transr=TR[tr], uplo=UL[ul])
    torch.cuda.synchronize()
    rel = ((I_our - I_ref).abs().max() / I_ref.abs().max()).item()
    assert rel <= 2e-4, rel


@pytest.mark.gpu
@pytest.mark.parametrize("tr,ul", VARIANTS)
@pytest.mark.parametrize("n,bad", [(200, 7), (200, 150)])
def test_info_vs_reference(curfp, ref, orc, tr, ul, n, bad):
    M = np.eye(n) * 2.0
    M[bad - 1, bad - 1] = -3.0
    arf = orc.strttf(tr, ul, n, M).astype(np.float32)
    a1, a2 = dev(arf), dev(arf)
    st, info_ref = ref.spftrf(tr, ul, n, a1)
    assert st == 0
    assert curfp.spftrf(a2, transr=TR[tr], uplo=UL[ul], check=False) == info_ref == bad


@pytest.mark.gpu
@pytest.mark.parametrize("n,m", [(1, 4), (64, 3), (65, 17), (1000, 64), (1001, 1)])
@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_ssfmm_vs_reference(curfp, ref, n, m, side, tr, ul):
    """Same RFP matrix and operands through both libraries' curfpSsfmm:
    agreement to FP32 summation-order spread (max-abs 2e-5 of the scale)."""
    g = torch.Generator(device="cuda").manual_seed(n + 7 * m + side)
    arf = torch.randn(n * (n + 1) // 2, device="cuda", generator=g)
    rows, cols = (n, m) if side == 0 else (m, n)
    B = torch.randn(cols, rows, device="cuda", generator=g)  # column-major rows x cols
    C0 = torch.randn(cols, rows, device="cuda", generator=g)
    C_ref, C_our = C0.clone(), C0.clone()
    assert ref.ssfmm(tr, ul, side, rows, cols, 0.75, arf, B, rows, -0.5, C_ref, rows) == 0
    curfp.ssfmm_raw(curfp._get_handle(), tr, ul, side, rows, cols, 0.75, arf, B, rows, -0.5,
                    C_our, rows)
    torch.cuda.synchronize()
    scale = C_ref.abs().max().item()
    assert (C_our - C_ref).abs().max().item() <= 2e-5 * scale * max(1.0, n ** 0.5 / 8)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 65, 1000, 1001])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_ssfmv_and_norms_vs_reference(curfp, ref, n, tr, ul):
    g = torch.Generator(device="cuda").manual_seed(n + 3)
    arf = torch.randn(n * (n + 1) // 2, device="cuda", generator=g)
    x = torch.randn(n, device="cuda", generator=g)
    y0 = torch.randn(n, device="cuda", generator=g)
    y_ref, y_our = y0.clone(), y0.clone()
    assert ref.ssfmv(tr, ul, n, 1.5, arf, x, 1, 0.25, y_ref, 1) == 0
    curfp.ssfmv(arf, x, y_our, alpha=1.5, beta=0.25, transr=TR[tr], uplo=UL[ul])
    torch.cuda.synchronize()
    scale = y_ref.abs().max().item()
    assert (y_our - y_ref).abs().max().item() <= 2e-5 * scale * max(1.0, n ** 0.5 / 8)
    for norm, s in ((0, "M"), (1, "1"), (2, "F")):
        st, want = ref.slansf(norm, tr, ul, n, arf)
        assert st == 0
        got = curfp.slansf(arf, s, transr=TR[tr], uplo=UL[ul])
        assert abs(got - want) <= 1e-5 * want, (s, got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 3, 64, 300, 1001])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_spfcon_vs_reference(curfp, ref, n, tr, ul):
    """Both estimators on the same factor: the same iteration (argmax picks
    and stopping) gives the same estimate up to FP32 solve differences."""
    g = torch.Generator(device="cuda").manual_seed(n + 11)
    A = torch.randn(n, max(1, n // 4), device="cuda", generator=g)
    C = torch.empty(n * (n + 1) // 2, device="cuda")
    curfp.ssfrk(A, C, alpha=1.0 / max(1, n // 4), transr=TR[tr], uplo=UL[ul])
    curfp.add_to_diagonal(C, 0.05, transr=TR[tr], uplo=UL[ul])
    anorm = curfp.slansf(C, "1", transr=TR[tr], uplo=UL[ul])
    assert curfp.spftrf(C, transr=TR[tr], uplo=UL[ul]) == 0
    st, want = ref.spfcon(tr, ul, n, C, anorm)
    assert st == 0
    got = curfp.spfcon(C, anorm, transr=TR[tr], uplo=UL[ul])
    assert abs(got - want) <= 1e-3 * want, (got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 65, 1000, 1001])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_ssfr_ssfr2_vs_reference(curfp, ref, n, tr, ul):
    g = torch.Generator(device="cuda").manual_seed(n + 17)
    arf = torch.randn(n * (n + 1) // 2, device="cuda", generator=g)
    x = torch.randn(n, device="cuda", generator=g)
    y = torch.randn(n, device="cuda", generator=g)
    a_ref, a_our = arf.clone(), arf.clone()
    assert ref.ssfr(tr, ul, n, 0.75, x, 1, a_ref) == 0
    curfp.ssfr(a_our, x, alpha=0.75, transr=TR[tr], uplo=UL[ul])
    torch.cuda.synchronize()
    assert (a_our - a_ref).abs().max().item() <= 1e-6 * a_ref.abs().max().item()
    assert ref.ssfr2(tr, ul, n, -0.5, x, 1, y, 1, a_ref) == 0
    curfp.ssfr2(a_our, x, y, alpha=-0.5, transr=TR[tr], uplo=UL[ul])
    torch.cuda.synchronize()
    assert (a_our - a_ref).abs().max().item() <= 2e-6 * a_ref.abs().max().item()


@pytest.mark.gpu
@pytest.mark.parametrize("n,k", [(65, 32), (1000, 128), (1001, 128)])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_double_pipeline_vs_reference(curfp, ref, n, k, tr, ul):
    """The FP64 twins against the reference's own curfpD* routines (cuBLAS /
    cuSOLVER in FP64) on the same inputs: agreement to FP64 summation-order
    spread (1e-12 relative on O(1) data, cond ~ 45)."""
    g = torch.Generator(device="cuda").manual_seed(n + 5 * tr + ul)
    A = torch.randn(n, k, device="cuda", dtype=torch.float64, generator=g) / k ** 0.5
    nt = n * (n + 1) // 2
    C_ref = torch.empty(nt, device="cuda", dtype=torch.float64)
    C_our = torch.empty_like(C_ref)
    assert ref.dsfrk(tr, ul, 1, n, k, 1.0, A, k, 0.0, C_ref) == 0
    curfp.dsfrk(A, C_our, transr=TR[tr], uplo=UL[ul])
    torch.cuda.synchronize()
    assert (C_our - C_ref).abs().max().item() <= 1e-13
    curfp.add_to_diagonal(C_ref, 1.0, transr=TR[tr], uplo=UL[ul])
    C_our.copy_(C_ref)
    st, info = ref.dpftrf(tr, ul, n, C_ref)
    assert st == 0 and info == 0
    assert curfp.dpftrf(C_our, transr=TR[tr], uplo=UL[ul]) == 0
    assert ((C_our - C_ref).abs().max() / C_ref.abs().max()).item() <= 1e-12
    B = torch.randn(8, n, device="cuda", dtype=torch.float64, generator=g)
    X_ref, X_our = B.clone(), B.clone()
    assert ref.dpftrs(tr, ul, n, 8, C_ref, X_ref, n) == 0
    curfp.dpftrs_raw(curfp._get_handle(), tr, ul, n, 8, C_our, X_our, n)
    torch.cuda.synchronize()
    assert ((X_our - X_ref).abs().max() / X_ref.abs().max()).item() <= 1e-12
    I_ref, I_our = C_ref.clone(), C_our.clone()
    assert ref.dpftri(tr, ul, n, I_ref) == 0
    curfp.dpftri(I_our, transr=TR[tr], uplo=UL[ul])
    torch.cuda.synchronize()
    assert ((I_our - I_ref).abs().max() / I_ref.abs().max()).item() <= 1e-12
