"""curfpSpftrsNoAlloc: the RFP solve for callers that cannot let the library
allocate device memory while they run -- a process whose GPU memory is owned
by another allocator, or a loop where a cudaMalloc (which may synchronise the
device or fail under memory pressure) is not acceptable.  Its scratch lives in
a static device array, so it is limited to n <= 16384 and nrhs <= 512.

Checked through the C ABI against curfpSpftrs on the same factor, on two
calls in a row (the static array keeps the previous call's contents), within
the solve tolerance used elsewhere in the tests.  This file is collected last
so that a run stopping at the first failure has already run every other
test; it also passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest
import torch

from conftest import VARIANTS

RTOL = 1e-5


def _solve(lib, h, fn, tr, ul, n, nrhs, F, B):
    X = B.clone()
    st = getattr(lib, fn)(h.ptr, tr, ul, n, nrhs, ctypes.c_void_p(F.data_ptr()),
                          ctypes.c_void_p(X.data_ptr()), n)
    torch.cuda.synchronize()
    assert st == 0, (fn, st)
    return X


@pytest.mark.gpu
@pytest.mark.parametrize("n,nrhs", [(3001, 7), (4096, 64), (16384, 64), (1000, 512)])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_no_alloc_matches_spftrs(curfp, n, nrhs, tr, ul):
    k = max(8, n // 32)
    g = torch.Generator(device="cuda").manual_seed(n + 10 * tr + ul)
    A = torch.randn(n, k, device="cuda", generator=g) / k ** 0.5
    C = torch.empty(n * (n + 1) // 2, device="cuda")
    T, U = "NT"[tr], "LU"[ul]
    curfp.ssfrk(A, C, transr=T, uplo=U)
    curfp.add_to_diagonal(C, 1.0, transr=T, uplo=U)
    assert curfp.spftrf(C, transr=T, uplo=U) == 0
    B = torch.randn(nrhs, n, device="cuda", generator=g)  # column-major n x nrhs
    with curfp.Handle() as h:
        lib = h._lib
        ref = _solve(lib, h, "curfpSpftrs", tr, ul, n, nrhs, C, B)
        for _ in range(2):  # two calls in a row share the static scratch
            out = _solve(lib, h, "curfpSpftrsNoAlloc", tr, ul, n, nrhs, C, B)
            np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(),
                                       rtol=RTOL, atol=RTOL * ref.abs().max().item())


@pytest.mark.gpu
def test_no_alloc_rejects_sizes_beyond_limits(curfp):
    with curfp.Handle() as h:
        lib = h._lib
        null = ctypes.c_void_p(0)
        assert lib.curfpSpftrsNoAlloc(h.ptr, 1, 1, 16385, 1, null, null, 16385) == 3
        assert lib.curfpSpftrsNoAlloc(h.ptr, 1, 1, 100, 513, null, null, 100) == 3
        assert lib.curfpSpftrsNoAlloc(h.ptr, 1, 1, 0, 5, null, null, 1) == 0
