"""curfpSpftrfFromHost: factoring an RFP array that is in host memory.

The factor must equal curfpSpftrfEx's on a device copy of the same array bit
for bit (the same planner and kernels; only the order of the host-to-device
copy differs), for every storage variant, odd and even n, both math modes,
pinned and pageable host memory, with and without the device copy of the
original (which must equal the input bit for bit).  A matrix that is not
positive definite gives the same info and the same partial factor.
"""
import ctypes

import pytest
import torch

from conftest import VARIANTS
from helpers import TR, UL


def make(curfp, n, tr, ul, seed, shift):
    k = max(1, n // 4)
    g = torch.Generator(device="cuda").manual_seed(seed)
    A = torch.randn(n, k, device="cuda", generator=g) / k ** 0.5
    C = torch.empty(n * (n + 1) // 2, device="cuda")
    curfp.ssfrk(A, C, transr=TR[tr], uplo=UL[ul])
    curfp.add_to_diagonal(C, shift, transr=TR[tr], uplo=UL[ul])
    return C


def from_host(h, n, tr, ul, host, C, O, math):
    info = ctypes.c_int(-7)
    st = h._lib.curfpSpftrfFromHost(h.ptr, tr, ul, n, ctypes.c_void_p(host.data_ptr()),
                                    ctypes.c_void_p(C.data_ptr()),
                                    ctypes.c_void_p(O.data_ptr() if O is not None else 0),
                                    ctypes.byref(info), math)
    torch.cuda.synchronize()
    return st, info.value


CASES = [(n, tr, ul, m, shift)
         for n in (1, 2, 257, 1000, 4097)
         for tr, ul in VARIANTS
         for m in (0, 1)
         for shift in ((1.0, -2.0) if n == 1000 else (1.0,))]


@pytest.mark.gpu
@pytest.mark.parametrize("n,tr,ul,math,shift", CASES)
def test_from_host_matches_device_factor(curfp, n, tr, ul, math, shift):
    C0 = make(curfp, n, tr, ul, n + 2 * tr + ul, shift)
    h = curfp._get_handle()
    ref = C0.clone()
    info = ctypes.c_int()
    assert h._lib.curfpSpftrfEx(h.ptr, tr, ul, n, ctypes.c_void_p(ref.data_ptr()),
                                ctypes.byref(info), math) == 0
    torch.cuda.synchronize()
    ref_info = info.value
    if shift < 0:
        assert ref_info > 0
    for pinned in (True, False):
        host = C0.cpu()
        if pinned:
            host = host.pin_memory()
        for keep in (True, False):
            C = torch.full_like(C0, float("nan"))
            O = torch.full_like(C0, float("nan")) if keep else None
            st, inf = from_host(h, n, tr, ul, host, C, O, math)
            assert st == 0 and inf == ref_info, (st, inf, ref_info)
            assert torch.equal(C, ref)
            if keep:
                assert torch.equal(O, C0)


@pytest.mark.gpu
def test_from_host_python_wrapper(curfp):
    from curfp_b200 import precision as P
    n = 3001
    C0 = make(curfp, n, 1, 1, 5, 1.0)
    ref = C0.clone()
    P.spftrf(ref)
    C = torch.empty_like(C0)
    O = torch.empty_like(C0)
    assert P.spftrf_from_host(C0.cpu().pin_memory(), C, O) == 0
    torch.cuda.synchronize()
    assert torch.equal(C, ref) and torch.equal(O, C0)


@pytest.mark.gpu
def test_from_host_arguments(curfp):
    h = curfp._get_handle()
    n = 8
    host = torch.zeros(n * (n + 1) // 2)
    C = torch.zeros(n * (n + 1) // 2, device="cuda")
    info = ctypes.c_int()
    p = ctypes.c_void_p
    lib = h._lib
    # the factor and the original copy must differ; n >= 0; info; math 0/1
    assert lib.curfpSpftrfFromHost(h.ptr, 1, 1, n, p(host.data_ptr()), p(C.data_ptr()),
                                   p(C.data_ptr()), ctypes.byref(info), 1) == 3
    assert lib.curfpSpftrfFromHost(h.ptr, 1, 1, -1, p(host.data_ptr()), p(C.data_ptr()),
                                   None, ctypes.byref(info), 1) == 3
    assert lib.curfpSpftrfFromHost(h.ptr, 1, 1, n, p(host.data_ptr()), p(C.data_ptr()),
                                   None, None, 1) == 3
    assert lib.curfpSpftrfFromHost(h.ptr, 1, 1, n, p(host.data_ptr()), p(C.data_ptr()),
                                   None, ctypes.byref(info), 7) == 3
    assert lib.curfpSpftrfFromHost(None, 1, 1, n, p(host.data_ptr()), p(C.data_ptr()),
                                   None, ctypes.byref(info), 1) == 1
    assert lib.curfpSpftrfFromHost(h.ptr, 1, 1, 0, None, None, None, ctypes.byref(info),
                                   1) == 0 and info.value == 0
