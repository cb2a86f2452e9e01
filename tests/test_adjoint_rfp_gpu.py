"""The Cholesky adjoint in RFP layout (curfpSpftrfBackward: recursive
blocked algorithm, in place on the cotangent, no n x n scratch) at large n,
through two exact identities that need no dense FP64 reference:

* f = 1/2 ||L||_F^2 = 1/2 tr(A): with Lbar = L the cotangent of A's stored
  elements is 1/2 on the diagonal and 0 elsewhere.
* f = sum_i log L_ii = 1/2 log det A: with Lbar = diag(1/L_ii) it is A^-1
  off the diagonal and 1/2 diag(A^-1) on it; A^-1 comes from spftri on the
  same factor (an independent code path).

Stated bounds (A = X X^T + I, X ~ N(0,1)/sqrt(k), cond ~ 45): first identity
max |Abar - 1/2 I| <= 1e-4; second ||Abar - A^-1 (diag halved)||_F /
||A^-1||_F <= 5e-5 (both sides FP32 computations; spftri's own inverse
residual is ~1e-5 at n = 32768); both for all 8 variants at n = 8192 and two
at n = 32768, in both math modes of the solves.  The dense FP64 comparison at n = 8192 is
in test_autograd_gpu.py."""
import ctypes

import pytest
import torch

from conftest import VARIANTS
from helpers import TR, UL


def factor(curfp, n, tr, ul, seed):
    k = n // 32
    g = torch.Generator(device="cuda").manual_seed(seed)
    A = torch.randn(n, k, device="cuda", generator=g) / k ** 0.5
    C = torch.empty(n * (n + 1) // 2, device="cuda")
    curfp.ssfrk(A, C, transr=TR[tr], uplo=UL[ul])
    del A
    curfp.add_to_diagonal(C, 1.0, transr=TR[tr], uplo=UL[ul])
    assert curfp.spftrf(C, transr=TR[tr], uplo=UL[ul]) == 0
    return C


def backward(curfp, n, tr, ul, L, G, math):
    h = curfp._get_handle()
    st = h._lib.curfpSpftrfBackward(h.ptr, tr, ul, n, ctypes.c_void_p(L.data_ptr()),
                                    ctypes.c_void_p(G.data_ptr()), ctypes.c_void_p(G.data_ptr()),
                                    math)
    torch.cuda.synchronize()
    assert st == 0, st


CASES = [(8192, tr, ul, m) for tr, ul in VARIANTS for m in (0, 1)] + \
        [(32768, 1, 1, 1), (32768, 0, 0, 1)]


@pytest.mark.gpu
@pytest.mark.parametrize("n,tr,ul,math", CASES)
def test_adjoint_identities(curfp, n, tr, ul, math):
    L = factor(curfp, n, tr, ul, n + 2 * tr + ul)
    d = curfp.rfp_diag_indices(n, transr=TR[tr], uplo=UL[ul])
    # f = 1/2 tr(A)
    G = L.clone()
    backward(curfp, n, tr, ul, L, G, math)
    G[d] -= 0.5
    err1 = G.abs().max().item()
    assert err1 <= 1e-4, err1
    # f = 1/2 log det A
    G.zero_()
    G[d] = 1.0 / L[d]
    backward(curfp, n, tr, ul, L, G, math)
    Z = L.clone()
    curfp.spftri(Z, transr=TR[tr], uplo=UL[ul])
    Z[d] *= 0.5
    err2 = (torch.linalg.norm(G - Z) / torch.linalg.norm(Z)).item()
    assert err2 <= 5e-5, err2


@pytest.mark.gpu
def test_adjoint_rejects_output_aliasing_factor(curfp):
    n = 300
    L = factor(curfp, n, 1, 1, 3)
    h = curfp._get_handle()
    p = ctypes.c_void_p(L.data_ptr())
    assert h._lib.curfpSpftrfBackward(h.ptr, 1, 1, n, p, p, p, 0) == 3
