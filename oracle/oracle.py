"""ctypes front end of the plain-C FP64 oracle (oracle/rfp_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker the library is compared against.
Conventions follow the reference C ABI: enums as ints (transr/trans 0=N 1=T,
uplo 0=L 1=U), dense operands column-major with a leading dimension, except
strttf/stfttr whose full matrix is row-major (reference
src/curfp_strttf.cu:1-8).  Arrays are numpy float64; results are returned as
new arrays (inputs are not modified).
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "librfp_oracle.so"
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_I64 = ctypes.POINTER(ctypes.c_int64)
_i = ctypes.c_int
_d = ctypes.c_double


def build() -> Path:
    src = HERE / "rfp_oracle.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB))
        L.orc_ssfrk.argtypes = [_i, _i, _i, _i, _i, _d, _D, _i, _d, _D]
        L.orc_ssfr2k.argtypes = [_i, _i, _i, _i, _i, _d, _D, _i, _D, _i, _d, _D]
        L.orc_strttf.argtypes = [_i, _i, _i, _D, _i, _D]
        L.orc_stfttr.argtypes = [_i, _i, _i, _D, _D, _i]
        L.orc_diag_indices.argtypes = [_i, _i, _i, _I64]
        L.orc_spftrf.argtypes = [_i, _i, _i, _D]
        L.orc_spftrf.restype = _i
        L.orc_spftrs.argtypes = [_i, _i, _i, _i, _D, _D, _i]
        L.orc_spftri.argtypes = [_i, _i, _i, _D]
        L.orc_spftri.restype = _i
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())


def ssfrk(transr, uplo, trans, n, k, alpha, A, lda, beta, C):
    A = _f64(A) if A is not None else np.zeros(1)
    C = _f64(C).copy()
    lib().orc_ssfrk(transr, uplo, trans, n, k, alpha, _p(A), lda, beta, _p(C))
    return C


def ssfr2k(transr, uplo, trans, n, k, alpha, A, lda, B, ldb, beta, C):
    A, B, C = _f64(A), _f64(B), _f64(C).copy()
    lib().orc_ssfr2k(transr, uplo, trans, n, k, alpha, _p(A), lda, _p(B), ldb, beta, _p(C))
    return C


def strttf(transr, uplo, n, A_rowmajor, lda=None):
    A = _f64(A_rowmajor)
    arf = np.zeros(n * (n + 1) // 2)
    lib().orc_strttf(transr, uplo, n, _p(A), lda or n, _p(arf))
    return arf


def stfttr(transr, uplo, n, arf, lda=None):
    arf = _f64(arf)
    lda = lda or n
    A = np.zeros(n * lda)
    lib().orc_stfttr(transr, uplo, n, _p(arf), _p(A), lda)
    return A.reshape(n, lda)


def diag_indices(transr, uplo, n):
    out = np.zeros(n, dtype=np.int64)
    lib().orc_diag_indices(transr, uplo, n, out.ctypes.data_as(_I64))
    return out


def spftrf(transr, uplo, n, arf):
    a = _f64(arf).copy()
    info = lib().orc_spftrf(transr, uplo, n, _p(a))
    return a, info


def spftrs(transr, uplo, n, nrhs, arf, B_colmajor, ldb):
    a, b = _f64(arf), _f64(B_colmajor).copy()
    lib().orc_spftrs(transr, uplo, n, nrhs, _p(a), _p(b), ldb)
    return b


def spftri(transr, uplo, n, arf):
    a = _f64(arf).copy()
    rc = lib().orc_spftri(transr, uplo, n, _p(a))
    return a, rc


def rfp_to_dense_sym(transr, uplo, n, arf) -> np.ndarray:
    """Full symmetric n x n matrix represented by an RFP array."""
    T = stfttr(transr, uplo, n, arf)
    return T + np.triu(T, 1).T if uplo == 1 else T + np.tril(T, -1).T


def rfp_to_factor(transr, uplo, n, arf) -> np.ndarray:
    """Lower Cholesky factor L (A = L L^T) from an RFP factor array."""
    T = stfttr(transr, uplo, n, arf)
    return T.T.copy() if uplo == 1 else T
