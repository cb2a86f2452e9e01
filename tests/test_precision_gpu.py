"""Precision form on the GPU: split-BF16 tcgen05 contractions in ssfrk and
spftrf, FP64-residual refined solves.  Errors are measured against FP64
(torch float64 on the GPU).  Stated bounds: the split-BF16 ssfrk agrees with
the FP64 product to 2e-6 relative (FP32 level); the split-BF16 factor's
relative backward error is within 2x of the plain-FP32 factor's; the refined
solve's backward error is <= the plain FP32 solve's."""
import numpy as np
import pytest
import torch

from conftest import VARIANTS
from helpers import TR, UL, host


def dense_sym(curfp, C, tr, ul):
    M = curfp.stfttr(C, transr=tr, uplo=ul).double()
    return M + M.triu(1).T if ul == "U" else M + M.tril(-1).T


def factor_L(curfp, F, tr, ul):
    T = curfp.stfttr(F, transr=tr, uplo=ul).double()
    return T.T if ul == "U" else T


@pytest.mark.gpu
@pytest.mark.parametrize("n,k", [(1024, 512), (1100, 640), (2048, 300), (4095, 1024)])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_ssfrk_bf16x3_vs_fp64(curfp, n, k, tr, ul):
    from curfp_b200 import precision as P
    g = torch.Generator(device="cuda").manual_seed(n + k)
    A = torch.randn(n, k, device="cuda", generator=g) / k ** 0.5
    C0 = torch.randn(n * (n + 1) // 2, device="cuda", generator=g)
    C = C0.clone()
    P.ssfrk(A, C, alpha=0.75, beta=-0.5, transr=TR[tr], uplo=UL[ul])
    ref = C0.double().clone()
    Ad = A.double()
    full = 0.75 * Ad @ Ad.T
    mask = torch.ones(n, n, device="cuda", dtype=torch.bool)
    mask = mask.triu() if ul else mask.tril()
    D = curfp.stfttr(C, transr=TR[tr], uplo=UL[ul]).double()
    D0 = curfp.stfttr(C0, transr=TR[tr], uplo=UL[ul]).double()
    err = (D - (full - 0.5 * D0))[mask].abs().max().item()
    scale = (full.abs() + 0.5 * D0.abs())[mask].max().item()
    assert err / scale <= 2e-6, err / scale


@pytest.mark.gpu
@pytest.mark.parametrize("tr,ul", [(1, 1), (0, 0)])
def test_ssfrk_bf16x3_k_split(curfp, tr, ul):
    """A contraction whose staged planes exceed the 4 GiB staging budget
    (n = 16384, k = 36864: 4.9 GiB) runs as two k-slabs; C accumulates across
    them with beta applied once.  Checked on 256 sampled rows in FP64."""
    from curfp_b200 import precision as P
    from scale_lib import rfp_offsets
    n, k = 16384, 36864
    g = torch.Generator(device="cuda").manual_seed(k)
    A = torch.randn(n, k, device="cuda", generator=g) / k ** 0.5
    C0 = torch.randn(n * (n + 1) // 2, device="cuda", generator=g)
    C = C0.clone()
    P.ssfrk(A, C, alpha=0.75, beta=-0.5, transr=TR[tr], uplo=UL[ul])
    rows = torch.randperm(n, device="cuda", generator=g)[:256].sort().values
    offs = rfp_offsets(tr, ul, n, rows)
    Ad = A.double()
    want = 0.75 * (Ad[rows] @ Ad.T) - 0.5 * C0[offs].double()
    err = (C[offs].double() - want).abs().max().item()
    scale = (0.75 * (Ad[rows] @ Ad.T).abs() + 0.5 * C0[offs].double().abs()).max().item()
    assert err / scale <= 2e-6, err / scale


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1000, 2049, 4096])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_spftrf_bf16x3_backward_error(curfp, n, tr, ul):
    from curfp_b200 import precision as P
    k = max(32, n // 32)
    g = torch.Generator(device="cuda").manual_seed(3 * n)
    A = torch.randn(n, k, device="cuda", generator=g) / k ** 0.5
    C = torch.empty(n * (n + 1) // 2, device="cuda")
    curfp.ssfrk(A, C, transr=TR[tr], uplo=UL[ul])
    curfp.add_to_diagonal(C, 0.1, transr=TR[tr], uplo=UL[ul])
    Ad = dense_sym(curfp, C, TR[tr], UL[ul])
    F32, F16 = C.clone(), C.clone()
    assert curfp.spftrf(F32, transr=TR[tr], uplo=UL[ul]) == 0
    assert P.spftrf(F16, transr=TR[tr], uplo=UL[ul]) == 0
    e32 = []
    for F in (F32, F16):
        L = factor_L(curfp, F, TR[tr], UL[ul])
        e32.append((torch.linalg.norm(Ad - L @ L.T) / torch.linalg.norm(Ad)).item())
    assert e32[1] <= 2.0 * e32[0] + 1e-7, e32


@pytest.mark.gpu
@pytest.mark.parametrize("n", [2048, 4095])
@pytest.mark.parametrize("lam", [1e-1, 1e-3])
def test_refined_solve(curfp, n, lam):
    from curfp_b200 import precision as P
    k = n // 32
    g = torch.Generator(device="cuda").manual_seed(n)
    A = torch.randn(n, k, device="cuda", generator=g) / k ** 0.5
    C = torch.empty(n * (n + 1) // 2, device="cuda")
    P.ssfrk(A, C)
    curfp.add_to_diagonal(C, lam)
    F16, F32 = C.clone(), C.clone()
    assert P.spftrf(F16) == 0
    assert curfp.spftrf(F32) == 0
    B = torch.randn(n, 64, device="cuda", generator=g)
    X32 = B.clone()
    curfp.spftrs(F32, X32)
    X16 = B.clone()
    iters = P.spftrs_refined(C, F16, X16, max_iter=3)
    assert iters >= 1
    Ad = dense_sym(curfp, C, "T", "U")
    nA = torch.linalg.norm(Ad)

    def berr(X):
        R = B.double() - Ad @ X.double()
        return (torch.linalg.norm(R, dim=0) /
                (nA * torch.linalg.norm(X.double(), dim=0) +
                 torch.linalg.norm(B.double(), dim=0))).max().item()
    assert berr(X16) <= berr(X32), (berr(X16), berr(X32))


@pytest.mark.gpu
@pytest.mark.parametrize("n,nr", [(300, 7), (1000, 70), (4097, 64)])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_symm_acc64(curfp, orc, tr, ul, n, nr):
    """Single k pass (n = 300) and k split over CTAs with FP64 atomics
    (n = 1000, 4097), one and several 64-column blocks."""
    from curfp_b200 import precision as P
    rng = np.random.default_rng(2 + n)
    M = rng.standard_normal((n, n)).astype(np.float32)
    M = M + M.T
    arf = orc.strttf(tr, ul, n, M.astype(np.float64)).astype(np.float32)
    X = rng.standard_normal((n, nr)).astype(np.float32)
    Y = rng.standard_normal((n, nr)).astype(np.float32)
    out = P.ssfmm_acc64(torch.from_numpy(arf).cuda(), torch.from_numpy(X).cuda(),
                        torch.from_numpy(Y).cuda(), alpha=-1.0, beta=1.0,
                        transr=TR[tr], uplo=UL[ul])
    exp = Y.astype(np.float64) - M.astype(np.float64) @ X.astype(np.float64)
    # FP64 sums rounded once: within one FP32 rounding of the exact value
    np.testing.assert_allclose(host(out), exp, rtol=1.2e-7, atol=1e-30)


@pytest.mark.gpu
def test_precision_info(curfp, orc):
    from curfp_b200 import precision as P
    n = 1500
    M = np.eye(n) * 3.0
    M[1200, 1200] = -1.0
    C = torch.from_numpy(orc.strttf(1, 1, n, M).astype(np.float32)).cuda()
    assert P.spftrf(C, check=False) == 1201
