"""curfpSpftrsNoAlloc: the RFP solve for callers that cannot let the library
allocate device memory while they run -- a process whose GPU memory is owned
by another allocator, or a loop where a cudaMalloc (which may synchronise the
device or fail under memory pressure) is not acceptable.  Its scratch lives in
a static device array, so it is limited to n <= 16384 and nrhs <= 512.

Checked through the C ABI against curfpSpftrs on the same factor, on two
calls in a row (the static array keeps the previous call's contents), within
the solve tolerance used elsewhere in the tests, and against FP64: the solve
backward error max_j ||b_j - A x_j|| / (||A||_F ||x_j|| + ||b_j||) <= 2e-6.
The largest case (n = 16384, nrhs = 512) fills the flag area exactly.  A
fresh handle's calls leave the device's free memory unchanged.  This file is
collected last so that a run stopping at the first failure has already run
every other test; it also passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest
import torch

from conftest import VARIANTS

RTOL = 1e-5
BERR = 2e-6


def _solve(lib, h, fn, tr, ul, n, nrhs, F, B):
    X = B.clone()
    st = getattr(lib, fn)(h.ptr, tr, ul, n, nrhs, ctypes.c_void_p(F.data_ptr()),
                          ctypes.c_void_p(X.data_ptr()), n)
    torch.cuda.synchronize()
    assert st == 0, (fn, st)
    return X


def _factor(curfp, n, tr, ul, seed):
    k = max(8, n // 32)
    g = torch.Generator(device="cuda").manual_seed(seed)
    A = torch.randn(n, k, device="cuda", generator=g) / k ** 0.5
    C = torch.empty(n * (n + 1) // 2, device="cuda")
    T, U = "NT"[tr], "LU"[ul]
    curfp.ssfrk(A, C, transr=T, uplo=U)
    curfp.add_to_diagonal(C, 1.0, transr=T, uplo=U)
    C0 = C.clone()
    assert curfp.spftrf(C, transr=T, uplo=U) == 0
    return C0, C, g


def _backward_error(curfp, C0, tr, ul, B, X):
    """FP64 solve backward error; B and X hold the column-major n x nrhs
    blocks as (nrhs, n) row-major tensors."""
    M = curfp.stfttr(C0, transr="NT"[tr], uplo="LU"[ul]).double()
    S = M + M.triu(1).T if ul == 1 else M + M.tril(-1).T
    Xd, Bd = X.double().T, B.double().T
    R = Bd - S @ Xd
    den = torch.linalg.norm(S) * Xd.norm(dim=0) + Bd.norm(dim=0)
    return (R.norm(dim=0) / den).max().item()


@pytest.mark.gpu
@pytest.mark.parametrize("n,nrhs", [(3001, 7), (4096, 64), (16384, 64), (1000, 512),
                                    (16384, 512)])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_no_alloc_matches_spftrs(curfp, n, nrhs, tr, ul):
    C0, C, g = _factor(curfp, n, tr, ul, n + 10 * tr + ul)
    B = torch.randn(nrhs, n, device="cuda", generator=g)  # column-major n x nrhs
    with curfp.Handle() as h:
        lib = h._lib
        ref = _solve(lib, h, "curfpSpftrs", tr, ul, n, nrhs, C, B)
        for _ in range(2):  # two calls in a row share the static scratch
            out = _solve(lib, h, "curfpSpftrsNoAlloc", tr, ul, n, nrhs, C, B)
            np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(),
                                       rtol=RTOL, atol=RTOL * ref.abs().max().item())
    berr = _backward_error(curfp, C0, tr, ul, B, out)
    assert berr <= BERR, berr


@pytest.mark.gpu
def test_no_alloc_leaves_free_memory_unchanged(curfp):
    """Nothing is allocated on the call path: after one call has loaded the
    kernels (module loading may take memory once per process), the calls of a
    fresh handle leave the device's free memory as it was."""
    n, nrhs, tr, ul = 8000, 100, 1, 1
    C0, C, g = _factor(curfp, n, tr, ul, 99)
    B = torch.randn(nrhs, n, device="cuda", generator=g)
    with curfp.Handle() as warm:
        _solve(warm._lib, warm, "curfpSpftrsNoAlloc", tr, ul, n, nrhs, C, B)
    X = B.clone()
    with curfp.Handle() as h:
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        for _ in range(3):
            st = h._lib.curfpSpftrsNoAlloc(h.ptr, tr, ul, n, nrhs,
                                           ctypes.c_void_p(C.data_ptr()),
                                           ctypes.c_void_p(X.data_ptr()), n)
            assert st == 0, st
            X.copy_(B)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, (free0, free1)


@pytest.mark.gpu
def test_no_alloc_after_planted_wait_timeout(curfp):
    """The bounded-wait self-test sets the handle's kernel error word (code 5)
    and reports it through the check every routine with bounded waits runs;
    the next no-allocation solve on the same handle starts clean."""
    n, nrhs, tr, ul = 2000, 9, 0, 0
    C0, C, g = _factor(curfp, n, tr, ul, 5)
    B = torch.randn(nrhs, n, device="cuda", generator=g)
    with curfp.Handle() as h:
        code = ctypes.c_int(0)
        assert h._lib.curfpDiagWaitTimeout(h.ptr, ctypes.byref(code)) == 4
        assert code.value == 5
        X = _solve(h._lib, h, "curfpSpftrsNoAlloc", tr, ul, n, nrhs, C, B)
    assert _backward_error(curfp, C0, tr, ul, B, X) <= BERR


@pytest.mark.gpu
def test_no_alloc_rejects_sizes_beyond_limits(curfp):
    with curfp.Handle() as h:
        lib = h._lib
        null = ctypes.c_void_p(0)
        assert lib.curfpSpftrsNoAlloc(h.ptr, 1, 1, 16385, 1, null, null, 16385) == 3
        assert lib.curfpSpftrsNoAlloc(h.ptr, 1, 1, 100, 513, null, null, 100) == 3
        assert lib.curfpSpftrsNoAlloc(h.ptr, 1, 1, 0, 5, null, null, 1) == 0
