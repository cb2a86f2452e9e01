"""ssfmm / ssfmv / ssfr / ssfr2 on the GPU, all 8 variants (both sides for ssfmm),
against FP64 products of the dense symmetric matrix (oracle expansion of the RFP
array): max-abs error within 2e-6 of the scale times sqrt(n)/8 (FP32
summation).  Also: BLAS increments (negative, strided), alpha = 0 reads
neither A nor B, beta = 0 does not read C, argument errors."""
import numpy as np
import pytest
import torch

from conftest import VARIANTS
from helpers import TR, UL, dev, host


def tol(n):
    return 2e-6 * max(1.0, n ** 0.5 / 8) * 8


@pytest.mark.gpu
@pytest.mark.parametrize("n,m", [(1, 5), (2, 2), (63, 7), (64, 64), (65, 130), (999, 33),
                                 (2048, 256)])
@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_ssfmm_vs_fp64(curfp, orc, n, m, side, tr, ul):
    rng = np.random.default_rng(n * 3 + m + (side == "R"))
    nt = n * (n + 1) // 2
    arf = rng.standard_normal(nt).astype(np.float32)
    A = orc.rfp_to_dense_sym(tr, ul, n, arf.astype(np.float64))
    shape = (n, m) if side == "L" else (m, n)
    B = rng.standard_normal(shape).astype(np.float32)
    C = rng.standard_normal(shape).astype(np.float32)
    # the column-major kernel reads the storage of (rows, cols) tensors as
    # column-major rows x cols: hand it the transposes' storage
    Bt = dev(np.ascontiguousarray(B.T))
    Ct = dev(np.ascontiguousarray(C.T))
    rows, cols = shape
    curfp.ssfmm_raw(curfp._get_handle(), tr, ul, 0 if side == "L" else 1, rows, cols, 0.5,
                    dev(arf), Bt, rows, -1.5, Ct, rows)
    got = host(Ct).T.astype(np.float64)
    B64, C64 = B.astype(np.float64), C.astype(np.float64)
    want = 0.5 * (A @ B64 if side == "L" else B64 @ A) - 1.5 * C64
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= tol(n) * scale


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 3, 64, 65, 1000, 4097])
@pytest.mark.parametrize("tr,ul", VARIANTS)
@pytest.mark.parametrize("incx,incy", [(1, 1), (2, 3), (-1, 1), (3, -2)])
def test_ssfmv_vs_fp64(curfp, orc, n, tr, ul, incx, incy):
    rng = np.random.default_rng(n + 5 * abs(incx) + abs(incy) + 100)
    nt = n * (n + 1) // 2
    arf = rng.standard_normal(nt).astype(np.float32)
    A = orc.rfp_to_dense_sym(tr, ul, n, arf.astype(np.float64))
    xs = rng.standard_normal(n * abs(incx)).astype(np.float32)
    ys = rng.standard_normal(n * abs(incy)).astype(np.float32)
    # BLAS: element i at i*inc (inc > 0) or (n-1-i)*|inc| (inc < 0)
    ix = np.arange(n) * incx if incx > 0 else (n - 1 - np.arange(n)) * -incx
    iy = np.arange(n) * incy if incy > 0 else (n - 1 - np.arange(n)) * -incy
    x, y0 = xs[ix].astype(np.float64), ys[iy].astype(np.float64)
    yd = dev(ys)
    curfp.ssfmv_raw(curfp._get_handle(), tr, ul, n, 2.0, dev(arf), dev(xs), incx, 0.5, yd, incy)
    got = host(yd)
    want = 2.0 * A @ x + 0.5 * y0
    assert np.abs(got[iy] - want).max() <= tol(n) * np.abs(want).max()
    untouched = np.setdiff1d(np.arange(ys.size), iy)
    np.testing.assert_array_equal(got[untouched], ys[untouched])


@pytest.mark.gpu
def test_symm_alpha_beta_zero(curfp):
    n, m = 300, 20
    nan_a = torch.full((n * (n + 1) // 2,), float("nan"), device="cuda")
    nan_b = torch.full((m, n), float("nan"), device="cuda")
    C = torch.randn(m, n, device="cuda")
    want = 3.0 * C
    curfp.ssfmm_raw(curfp._get_handle(), 1, 1, 0, n, m, 0.0, nan_a, nan_b, n, 3.0, C, n)
    torch.testing.assert_close(C, want, rtol=0, atol=0)
    # beta = 0: C is written without being read
    A = torch.randn(n * (n + 1) // 2, device="cuda")
    B = torch.randn(m, n, device="cuda")
    C1 = torch.full((m, n), float("nan"), device="cuda")
    C2 = torch.zeros(m, n, device="cuda")
    curfp.ssfmm_raw(curfp._get_handle(), 1, 1, 0, n, m, 1.0, A, B, n, 0.0, C1, n)
    curfp.ssfmm_raw(curfp._get_handle(), 1, 1, 0, n, m, 1.0, A, B, n, 0.0, C2, n)
    torch.testing.assert_close(C1, C2, rtol=0, atol=0)
    y = curfp.ssfmv(A, torch.randn(n, device="cuda"))
    assert torch.isfinite(y).all()


@pytest.mark.gpu
def test_symm_argument_errors(curfp):
    h = curfp._get_handle()
    A = torch.zeros(10, device="cuda")
    B = torch.zeros(4, 4, device="cuda")
    with pytest.raises(RuntimeError, match="status=3"):
        curfp.ssfmm_raw(h, 1, 1, 0, 4, 4, 1.0, A, B, 3, 0.0, B, 4)  # ldb < m
    with pytest.raises(RuntimeError, match="status=3"):
        curfp.ssfmm_raw(h, 1, 1, 2, 4, 4, 1.0, A, B, 4, 0.0, B, 4)  # bad side
    with pytest.raises(RuntimeError, match="status=3"):
        curfp.ssfmv_raw(h, 1, 1, 4, 1.0, A, B, 0, 0.0, B, 1)  # incx = 0
    with pytest.raises(ValueError):
        curfp.ssfmm(A, torch.zeros(3, 4, device="cuda"))  # side L: A is 4 x 4, B has 3 rows


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 3, 64, 65, 1000, 4097])
@pytest.mark.parametrize("tr,ul", VARIANTS)
@pytest.mark.parametrize("incx,incy", [(1, 1), (2, -3)])
def test_ssfr_ssfr2_vs_fp64(curfp, orc, n, tr, ul, incx, incy):
    """Rank-1 / rank-2 updates of every stored element against FP64: one
    rounding of two FMAs per element (<= 2 ulp of the operand scale)."""
    rng = np.random.default_rng(n + abs(incy) + 7)
    nt = n * (n + 1) // 2
    arf = rng.standard_normal(nt).astype(np.float32)
    xs = rng.standard_normal(n * abs(incx)).astype(np.float32)
    ys = rng.standard_normal(n * abs(incy)).astype(np.float32)
    ix = np.arange(n) * incx if incx > 0 else (n - 1 - np.arange(n)) * -incx
    iy = np.arange(n) * incy if incy > 0 else (n - 1 - np.arange(n)) * -incy
    x, y = xs[ix].astype(np.float64), ys[iy].astype(np.float64)
    A = orc.rfp_to_dense_sym(tr, ul, n, arf.astype(np.float64))
    h = curfp._get_handle()
    a1 = dev(arf)
    curfp.ssfr_raw(h, tr, ul, n, 0.75, dev(xs), incx, a1)
    got = orc.rfp_to_dense_sym(tr, ul, n, host(a1).astype(np.float64))
    want = A + 0.75 * np.outer(x, x)
    assert np.abs(got - want).max() <= 4e-7 * max(1.0, np.abs(want).max())
    a2 = dev(arf)
    curfp.ssfr2_raw(h, tr, ul, n, -0.5, dev(xs), incx, dev(ys), incy, a2)
    got = orc.rfp_to_dense_sym(tr, ul, n, host(a2).astype(np.float64))
    want = A - 0.5 * (np.outer(x, y) + np.outer(y, x))
    assert np.abs(got - want).max() <= 6e-7 * max(1.0, np.abs(want).max())
    # alpha = 0: no-op, x not read
    a3 = dev(arf)
    curfp.ssfr_raw(h, tr, ul, n, 0.0, torch.full((n,), float("nan"), device="cuda"), 1, a3)
    np.testing.assert_array_equal(host(a3), arf)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [129, 20001])
@pytest.mark.parametrize("tr,ul", [(1, 1), (0, 0), (1, 0), (0, 1)])
def test_ssfmv_large_repeatable(curfp, n, tr, ul):
    """ssfmv against a dense FP64 torch product of the unpacked matrix
    (n = 20001: 2e8 stored elements, every 64 x 64 tile kind), and two calls
    agree bit for bit."""
    g = torch.Generator(device="cuda").manual_seed(n + tr + 2 * ul)
    M = torch.randn(n, n, device="cuda", generator=g)
    kw = dict(transr=TR[tr], uplo=UL[ul])
    arf = curfp.strttf(M, **kw)
    T = (M.triu() if ul else M.tril()).double()
    S = T + (T.triu(1).T if ul else T.tril(-1).T)
    del M, T
    x = torch.randn(n, device="cuda", generator=g)
    y0 = torch.randn(n, device="cuda", generator=g)
    y1, y2 = y0.clone(), y0.clone()
    curfp.ssfmv(arf, x, y1, alpha=-0.5, beta=2.0, **kw)
    curfp.ssfmv(arf, x, y2, alpha=-0.5, beta=2.0, **kw)
    assert torch.equal(y1, y2)
    want = -0.5 * (S @ x.double()) + 2.0 * y0.double()
    assert (y1.double() - want).abs().max().item() <= tol(n) * want.abs().max().item()
