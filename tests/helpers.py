"""Helpers shared by the GPU tests (imported by test modules only)."""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
REF_LIB = ROOT / "oracle" / "_ref" / "libcurfp_ref.so"
TR = {0: "N", 1: "T"}
UL = {0: "L", 1: "U"}


def dev(a, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def host(t) -> np.ndarray:
    return t.detach().cpu().numpy()


def rel_backward_error(orc, tr, ul, n, A_rfp, F_rfp) -> float:
    """||A - L L^T||_F / ||A||_F in FP64 from RFP arrays (n up to a few 1000)."""
    A = orc.rfp_to_dense_sym(tr, ul, n, np.asarray(A_rfp, np.float64))
    L = orc.rfp_to_factor(tr, ul, n, np.asarray(F_rfp, np.float64))
    return float(np.linalg.norm(A - L @ L.T) / np.linalg.norm(A))


def solve_backward_error(orc, tr, ul, n, A_rfp, X, B) -> float:
    """max_j ||b_j - A x_j|| / (||A|| ||x_j|| + ||b_j||) in FP64 (2-norms)."""
    A = orc.rfp_to_dense_sym(tr, ul, n, np.asarray(A_rfp, np.float64))
    X = np.asarray(X, np.float64)
    B = np.asarray(B, np.float64)
    R = B - A @ X
    nA = np.linalg.norm(A, 2) if n <= 2048 else np.linalg.norm(A)
    return float(np.max(np.linalg.norm(R, axis=0) /
                        (nA * np.linalg.norm(X, axis=0) + np.linalg.norm(B, axis=0))))


class RefLib:
    """The unmodified reference library (oracle/_ref, built by
    `make -C oracle ref`) called through its own C ABI."""

    def __init__(self):
        self.lib = ctypes.CDLL(str(REF_LIB))
        self.h = ctypes.c_void_p()
        assert self.lib.curfpCreate(ctypes.byref(self.h)) == 0

    def ssfrk(self, tr, ul, trans, n, k, alpha, A, lda, beta, C):
        a, b = ctypes.c_float(alpha), ctypes.c_float(beta)
        return self.lib.curfpSsfrk(self.h, tr, ul, trans, n, k, ctypes.byref(a),
                                   ctypes.c_void_p(A.data_ptr()), lda, ctypes.byref(b),
                                   ctypes.c_void_p(C.data_ptr()))

    def spftrf(self, tr, ul, n, C):
        info = ctypes.c_int(0)
        st = self.lib.curfpSpftrf(self.h, tr, ul, n, ctypes.c_void_p(C.data_ptr()),
                                  ctypes.byref(info))
        return st, info.value

    def spftrs(self, tr, ul, n, nrhs, C, B, ldb):
        return self.lib.curfpSpftrs(self.h, tr, ul, n, nrhs, ctypes.c_void_p(C.data_ptr()),
                                    ctypes.c_void_p(B.data_ptr()), ldb)

    def spftri(self, tr, ul, n, C):
        return self.lib.curfpSpftri(self.h, tr, ul, n, ctypes.c_void_p(C.data_ptr()))

    def strttf(self, tr, ul, n, A, lda, arf):
        return self.lib.curfpSstrttf(self.h, tr, ul, n, ctypes.c_void_p(A.data_ptr()), lda,
                                     ctypes.c_void_p(arf.data_ptr()))

    def stfttr(self, tr, ul, n, arf, A, lda):
        return self.lib.curfpSstfttr(self.h, tr, ul, n, ctypes.c_void_p(arf.data_ptr()),
                                     ctypes.c_void_p(A.data_ptr()), lda)

    def ssfmm(self, tr, ul, side, m, n, alpha, arf, B, ldb, beta, C, ldc):
        a, b = ctypes.c_float(alpha), ctypes.c_float(beta)
        return self.lib.curfpSsfmm(self.h, tr, ul, side, m, n, ctypes.byref(a),
                                   ctypes.c_void_p(arf.data_ptr()), ctypes.c_void_p(B.data_ptr()),
                                   ldb, ctypes.byref(b), ctypes.c_void_p(C.data_ptr()), ldc)

    def ssfmv(self, tr, ul, n, alpha, arf, x, incx, beta, y, incy):
        a, b = ctypes.c_float(alpha), ctypes.c_float(beta)
        return self.lib.curfpSsfmv(self.h, tr, ul, n, ctypes.byref(a),
                                   ctypes.c_void_p(arf.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                   incx, ctypes.byref(b), ctypes.c_void_p(y.data_ptr()), incy)

    def slansf(self, norm, tr, ul, n, arf):
        out = ctypes.c_float(0.0)
        st = self.lib.curfpSlansf(self.h, norm, tr, ul, n, ctypes.c_void_p(arf.data_ptr()),
                                  ctypes.byref(out))
        return st, out.value

    def spfcon(self, tr, ul, n, arf, anorm):
        out = ctypes.c_float(0.0)
        st = self.lib.curfpSpfcon(self.h, tr, ul, n, ctypes.c_void_p(arf.data_ptr()),
                                  ctypes.c_float(anorm), ctypes.byref(out))
        return st, out.value

    def ssfr(self, tr, ul, n, alpha, x, incx, arf):
        a = ctypes.c_float(alpha)
        return self.lib.curfpSsfr(self.h, tr, ul, n, ctypes.byref(a), ctypes.c_void_p(x.data_ptr()),
                                  incx, ctypes.c_void_p(arf.data_ptr()))

    def ssfr2(self, tr, ul, n, alpha, x, incx, y, incy, arf):
        a = ctypes.c_float(alpha)
        return self.lib.curfpSsfr2(self.h, tr, ul, n, ctypes.byref(a),
                                   ctypes.c_void_p(x.data_ptr()), incx,
                                   ctypes.c_void_p(y.data_ptr()), incy,
                                   ctypes.c_void_p(arf.data_ptr()))

    def dsfrk(self, tr, ul, trans, n, k, alpha, A, lda, beta, C):
        a, b = ctypes.c_double(alpha), ctypes.c_double(beta)
        return self.lib.curfpDsfrk(self.h, tr, ul, trans, n, k, ctypes.byref(a),
                                   ctypes.c_void_p(A.data_ptr()), lda, ctypes.byref(b),
                                   ctypes.c_void_p(C.data_ptr()))

    def dpftrf(self, tr, ul, n, C):
        info = ctypes.c_int(0)
        st = self.lib.curfpDpftrf(self.h, tr, ul, n, ctypes.c_void_p(C.data_ptr()),
                                  ctypes.byref(info))
        return st, info.value

    def dpftrs(self, tr, ul, n, nrhs, C, B, ldb):
        return self.lib.curfpDpftrs(self.h, tr, ul, n, nrhs, ctypes.c_void_p(C.data_ptr()),
                                    ctypes.c_void_p(B.data_ptr()), ldb)

    def dpftri(self, tr, ul, n, C):
        return self.lib.curfpDpftri(self.h, tr, ul, n, ctypes.c_void_p(C.data_ptr()))
