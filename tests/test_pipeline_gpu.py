"""Plain-FP32 pipeline at the CPU-runnable configuration: n in {4095, 4096},
k = 128, A ~ N(0,1)/sqrt(k), C = A A^T + 1.0 I in RFP (transr='T', uplo='U'),
spftrf, spftrs with 64 right-hand sides; accuracy against FP64.

Bounds (stated): relative backward error of the factor
||A - L L^T||_F / ||A||_F <= 2e-6, and solve backward error
max_j ||b - A x|| / (||A|| ||x|| + ||b||) <= 2e-6 (Frobenius ||A||).
FP32 unit roundoff is 6e-8; a stable Cholesky/solve stays within a small
multiple of sqrt(n)*eps on this well-conditioned (cond ~ 45) matrix."""
import numpy as np
import pytest
import torch

from helpers import RefLib, REF_LIB, TR, UL, dev, host


def fp64_errors(curfp, n, C0, F, X, B, tr="T", ul="U"):
    """Backward errors computed on the GPU in FP64 from unpacked matrices."""
    A = curfp.stfttr(C0, transr=tr, uplo=ul).double()
    A = A + A.triu(1).T if ul == "U" else A + A.tril(-1).T
    T = curfp.stfttr(F, transr=tr, uplo=ul).double()
    L = T.T if ul == "U" else T
    e_fac = (torch.linalg.norm(A - L @ L.T) / torch.linalg.norm(A)).item()
    R = B.double() - A @ X.double()
    nA = torch.linalg.norm(A)
    e_sol = (torch.linalg.norm(R, dim=0) /
             (nA * torch.linalg.norm(X.double(), dim=0) + torch.linalg.norm(B.double(), dim=0))).max().item()
    return e_fac, e_sol


@pytest.mark.gpu
@pytest.mark.parametrize("n", [4095, 4096])
@pytest.mark.parametrize("tr,ul", [("T", "U"), ("N", "L"), ("N", "U"), ("T", "L")])
def test_c1_pipeline(curfp, n, tr, ul):
    k = 128
    g = torch.Generator(device="cuda").manual_seed(n)
    A = torch.randn(n, k, device="cuda", generator=g) / k ** 0.5
    B = torch.randn(n, 64, device="cuda", generator=g)
    C = torch.empty(n * (n + 1) // 2, device="cuda")
    curfp.ssfrk(A, C, transr=tr, uplo=ul)
    curfp.add_to_diagonal(C, 1.0, transr=tr, uplo=ul)
    C0 = C.clone()
    assert curfp.spftrf(C, transr=tr, uplo=ul) == 0
    X = B.clone()
    curfp.spftrs(C, X, transr=tr, uplo=ul)
    e_fac, e_sol = fp64_errors(curfp, n, C0, C, X, B, tr, ul)
    assert e_fac <= 2e-6, e_fac
    assert e_sol <= 2e-6, e_sol
    # ssfrk against an FP64 product
    Cd = curfp.stfttr(C0, transr=tr, uplo=ul).double()
    Ad = A.double()
    full = Ad @ Ad.T + torch.eye(n, device="cuda", dtype=torch.float64)
    mask = torch.ones(n, n, device="cuda", dtype=torch.bool)
    mask = mask.triu() if ul == "U" else mask.tril()
    assert (Cd - full)[mask].abs().max().item() <= 1e-5


@pytest.mark.gpu
@pytest.mark.skipif(not REF_LIB.exists(), reason="reference build missing")
@pytest.mark.parametrize("n", [4095, 4096])
def test_c1_backward_error_not_worse_than_reference(curfp, n):
    """Same inputs through the reference GPU build: our factor and solve
    backward errors stay within 2x of the reference's."""
    ref = RefLib()
    k = 128
    g = torch.Generator(device="cuda").manual_seed(7 + n)
    A = torch.randn(n, k, device="cuda", generator=g) / k ** 0.5
    B = torch.randn(n, 64, device="cuda", generator=g)
    C = torch.empty(n * (n + 1) // 2, device="cuda")
    curfp.ssfrk(A, C)
    curfp.add_to_diagonal(C, 1.0)
    C0 = C.clone()
    Cr = C.clone()
    st, info = ref.spftrf(1, 1, n, Cr)
    assert st == 0 and info == 0
    Xr = B.t().contiguous()
    assert ref.spftrs(1, 1, n, 64, Cr, Xr, n) == 0
    torch.cuda.synchronize()
    curfp.spftrf(C)
    X = B.clone()
    curfp.spftrs(C, X)
    e_fac, e_sol = fp64_errors(curfp, n, C0, C, X, B)
    r_fac, r_sol = fp64_errors(curfp, n, C0, Cr, Xr.t(), B)
    assert e_fac <= 2 * r_fac + 1e-7, (e_fac, r_fac)
    assert e_sol <= 2 * r_sol + 1e-7, (e_sol, r_sol)
