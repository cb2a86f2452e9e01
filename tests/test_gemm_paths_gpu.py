"""The FP32 SIMT GEMM's two main loops give bitwise identical results.

Interior tiles of an unmasked product whose depth is a multiple of the k-tile
depth take the whole-tile loop (per-thread pointers advanced by a fixed step,
no bounds arithmetic); other tiles take the general loop (bounds checks and
zero fill per k-tile).  ssfrk in the FP32 math mode at k = 1000 (not a
multiple of 16 or 32: every tile takes the general loop) must equal ssfrk on
the same operand zero-padded to k = 1024 (interior tiles take the whole-tile
loop): the extra products are exact zeros and the FMA order is the same.
Both tile sizes (n = 600 fills fewer than 148 tiles of 128 and runs 64 x 64
tiles; n = 2300 runs 128 x 128), both transposes (row-contiguous and
k-contiguous operands), leading dimensions that allow 16-byte loads and odd
ones that do not, and all storage variants.
"""
import ctypes

import pytest
import torch

from conftest import VARIANTS

K, KPAD = 1000, 1024


def ssfrk(h, tr, ul, trans, n, k, A, lda, C, beta):
    one, b = ctypes.c_float(1.0), ctypes.c_float(beta)
    st = h._lib.curfpSsfrkEx(h.ptr, tr, ul, trans, n, k, ctypes.byref(one),
                             ctypes.c_void_p(A.data_ptr()), lda, ctypes.byref(b),
                             ctypes.c_void_p(C.data_ptr()), 0)
    assert st == 0


@pytest.mark.gpu
@pytest.mark.parametrize("n", [600, 2300])
@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("aligned", [True, False])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_whole_tile_loop_matches_general_loop(curfp, n, trans, aligned, tr, ul):
    h = curfp._get_handle()
    g = torch.Generator(device="cuda").manual_seed(n + 10 * trans + 100 * tr + 1000 * ul)
    if trans == 0:  # A is n x k, column-major, lda >= n
        lda = (n + 3) // 4 * 4 if aligned else n + 1  # n is even: n + 1 is odd
        buf = torch.zeros(KPAD * lda, device="cuda")
        view = buf.view(KPAD, lda)
        view[:K, :n] = torch.randn(K, n, device="cuda", generator=g)
    else:  # A is k x n, column-major, lda >= k
        lda = KPAD if aligned else KPAD + 1
        buf = torch.zeros(n * lda, device="cuda")
        view = buf.view(n, lda)
        view[:, :K] = torch.randn(n, K, device="cuda", generator=g)
    C0 = torch.randn(n * (n + 1) // 2, device="cuda", generator=g)
    C_general, C_whole = C0.clone(), C0.clone()
    ssfrk(h, tr, ul, trans, n, K, buf, lda, C_general, 0.5)
    ssfrk(h, tr, ul, trans, n, KPAD, buf, lda, C_whole, 0.5)
    torch.cuda.synchronize()
    assert torch.equal(C_general, C_whole)
    # and the result is the product (loose FP32 check against FP64)
    Ad = view[:K, :n].double().t() if trans == 0 else view[:, :K].double()
    full = (Ad @ Ad.t()).float().contiguous()  # symmetric: either triangle
    ref = curfp.strttf(full, transr="NT"[tr], uplo="LU"[ul]).double() + 0.5 * C0.double()
    err = ((C_whole.double() - ref).abs().max() / ref.abs().max()).item()
    assert err < 1e-5, err
