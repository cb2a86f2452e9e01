"""FP64 (D-prefix) twins of the RFP routines, mirroring the reference's
``curfp.d*`` functions (curfp/__init__.py:1347-2090): same names, keyword
arguments, defaults and errors as their S counterparts, float64 tensors."""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import check

_d = ctypes.c_double


def _validate64(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if t.dtype != torch.float64:
        raise ValueError(f"{name} must be float64 (got {t.dtype})")


def _pkg():
    from . import _get_handle, _fill, _hp, _n_from_rfp, _norm, _op, _ptr, _side
    return _get_handle, _fill, _hp, _n_from_rfp, _norm, _op, _ptr, _side


def _L():
    return _lib.load()


# --- raw API ----------------------------------------------------------------

def dsfrk_raw(handle, transr: int, uplo: int, trans: int, n: int, k: int, alpha: float,
              A: torch.Tensor, lda: int, beta: float, C: torch.Tensor) -> None:
    _, _, _hp, _, _, _, _ptr, _ = _pkg()
    if A is not None:
        _validate64(A, "A")
    _validate64(C, "C")
    a, b = _d(alpha), _d(beta)
    check(_L().curfpDsfrk(_hp(handle), transr, uplo, trans, n, k, ctypes.byref(a), _ptr(A), lda,
                          ctypes.byref(b), _ptr(C)))


def dpftrf_raw(handle, transr: int, uplo: int, n: int, A: torch.Tensor) -> int:
    _, _, _hp, _, _, _, _ptr, _ = _pkg()
    _validate64(A, "A")
    info = ctypes.c_int(0)
    check(_L().curfpDpftrf(_hp(handle), transr, uplo, n, _ptr(A), ctypes.byref(info)))
    return info.value


def dpftrs_raw(handle, transr: int, uplo: int, n: int, nrhs: int, A: torch.Tensor,
               B: torch.Tensor, ldb: int) -> None:
    _, _, _hp, _, _, _, _ptr, _ = _pkg()
    _validate64(A, "A")
    _validate64(B, "B")
    check(_L().curfpDpftrs(_hp(handle), transr, uplo, n, nrhs, _ptr(A), _ptr(B), ldb))


def dpftri_raw(handle, transr: int, uplo: int, n: int, A: torch.Tensor) -> None:
    _, _, _hp, _, _, _, _ptr, _ = _pkg()
    _validate64(A, "A")
    check(_L().curfpDpftri(_hp(handle), transr, uplo, n, _ptr(A)))


def dstrttf_raw(handle, transr: int, uplo: int, n: int, A: torch.Tensor, lda: int,
                arf: torch.Tensor) -> None:
    _, _, _hp, _, _, _, _ptr, _ = _pkg()
    _validate64(A, "A")
    _validate64(arf, "arf")
    check(_L().curfpDstrttf(_hp(handle), transr, uplo, n, _ptr(A), lda, _ptr(arf)))


def dstfttr_raw(handle, transr: int, uplo: int, n: int, arf: torch.Tensor, A: torch.Tensor,
                lda: int) -> None:
    _, _, _hp, _, _, _, _ptr, _ = _pkg()
    _validate64(arf, "arf")
    _validate64(A, "A")
    check(_L().curfpDstfttr(_hp(handle), transr, uplo, n, _ptr(arf), _ptr(A), lda))


def dsfr2k_raw(handle, transr: int, uplo: int, trans: int, n: int, k: int, alpha: float,
               A: torch.Tensor, lda: int, B: torch.Tensor, ldb: int, beta: float,
               C: torch.Tensor) -> None:
    _, _, _hp, _, _, _, _ptr, _ = _pkg()
    _validate64(A, "A")
    _validate64(B, "B")
    _validate64(C, "C")
    a, b = _d(alpha), _d(beta)
    check(_L().curfpDsfr2k(_hp(handle), transr, uplo, trans, n, k, ctypes.byref(a), _ptr(A),
                           lda, _ptr(B), ldb, ctypes.byref(b), _ptr(C)))


def dlansf_raw(handle, norm: int, transr: int, uplo: int, n: int, C: torch.Tensor) -> float:
    _, _, _hp, _, _, _, _ptr, _ = _pkg()
    _validate64(C, "C")
    out = _d(0.0)
    check(_L().curfpDlansf(_hp(handle), norm, transr, uplo, n, _ptr(C), ctypes.byref(out)))
    return float(out.value)


def dpfcon_raw(handle, transr: int, uplo: int, n: int, C: torch.Tensor, anorm: float) -> float:
    _, _, _hp, _, _, _, _ptr, _ = _pkg()
    _validate64(C, "C")
    out = _d(0.0)
    check(_L().curfpDpfcon(_hp(handle), transr, uplo, n, _ptr(C), _d(anorm), ctypes.byref(out)))
    return float(out.value)


def dsfmv_raw(handle, transr: int, uplo: int, n: int, alpha: float, arf: torch.Tensor,
              x: torch.Tensor, incx: int, beta: float, y: torch.Tensor, incy: int) -> None:
    _, _, _hp, _, _, _, _ptr, _ = _pkg()
    for t, nm in ((arf, "arf"), (x, "x"), (y, "y")):
        _validate64(t, nm)
    a, b = _d(alpha), _d(beta)
    check(_L().curfpDsfmv(_hp(handle), transr, uplo, n, ctypes.byref(a), _ptr(arf), _ptr(x),
                          incx, ctypes.byref(b), _ptr(y), incy))


def dsfmm_raw(handle, transr: int, uplo: int, side: int, m: int, n: int, alpha: float,
              arf: torch.Tensor, B: torch.Tensor, ldb: int, beta: float, C: torch.Tensor,
              ldc: int) -> None:
    _, _, _hp, _, _, _, _ptr, _ = _pkg()
    for t, nm in ((arf, "arf"), (B, "B"), (C, "C")):
        _validate64(t, nm)
    a, b = _d(alpha), _d(beta)
    check(_L().curfpDsfmm(_hp(handle), transr, uplo, side, m, n, ctypes.byref(a), _ptr(arf),
                          _ptr(B), ldb, ctypes.byref(b), _ptr(C), ldc))


def dsfr_raw(handle, transr: int, uplo: int, n: int, alpha: float, x: torch.Tensor, incx: int,
             arf: torch.Tensor) -> None:
    _, _, _hp, _, _, _, _ptr, _ = _pkg()
    _validate64(x, "x")
    _validate64(arf, "arf")
    a = _d(alpha)
    check(_L().curfpDsfr(_hp(handle), transr, uplo, n, ctypes.byref(a), _ptr(x), incx,
                         _ptr(arf)))


def dsfr2_raw(handle, transr: int, uplo: int, n: int, alpha: float, x: torch.Tensor, incx: int,
              y: torch.Tensor, incy: int, arf: torch.Tensor) -> None:
    _, _, _hp, _, _, _, _ptr, _ = _pkg()
    for t, nm in ((x, "x"), (y, "y"), (arf, "arf")):
        _validate64(t, nm)
    a = _d(alpha)
    check(_L().curfpDsfr2(_hp(handle), transr, uplo, n, ctypes.byref(a), _ptr(x), incx,
                          _ptr(y), incy, _ptr(arf)))


# --- tensor API ---------------------------------------------------------------

def dsfrk(A: torch.Tensor, C: torch.Tensor, *, alpha: float = 1.0, beta: float = 0.0,
          transr: str = "T", uplo: str = "U", trans: str = "T", n: int = None, k: int = None,
          lda: int = None) -> None:
    """C := alpha*A@A.T + beta*C (trans='T', A row-major n x k) in RFP, float64."""
    _get_handle, _fill, _, _n_from_rfp, _, _op, _, _ = _pkg()
    _validate64(A, "A")
    _validate64(C, "C")
    if n is None:
        n = _n_from_rfp(C.numel())
    tu = trans.upper()
    if k is None:
        k = A.shape[1] if tu == "T" else A.shape[0]
    if lda is None:
        lda = A.shape[1] if tu == "T" else A.shape[0]
    dsfrk_raw(_get_handle(), _op(transr), _fill(uplo), _op(trans), n, k, alpha, A, lda, beta, C)


def dpftrf(C: torch.Tensor, *, n: int = None, transr: str = "T", uplo: str = "U",
           check: bool = True) -> int:
    """In-place float64 RFP Cholesky; returns info."""
    _get_handle, _fill, _, _n_from_rfp, _, _op, _, _ = _pkg()
    _validate64(C, "C")
    if n is None:
        n = _n_from_rfp(C.numel())
    info = dpftrf_raw(_get_handle(), _op(transr), _fill(uplo), n, C)
    if check and info != 0:
        raise torch.linalg.LinAlgError(
            f"dpftrf: matrix is not positive definite "
            f"(leading minor of order {info} is not positive definite)")
    return info


def dpftrs(C: torch.Tensor, B: torch.Tensor, *, n: int = None, nrhs: int = None,
           transr: str = "T", uplo: str = "U") -> None:
    """Solve A X = B with the float64 RFP factor C; B (n, nrhs) or (n,) in place."""
    _get_handle, _fill, _, _n_from_rfp, _, _op, _, _ = _pkg()
    _validate64(C, "C")
    _validate64(B, "B")
    if n is None:
        n = _n_from_rfp(C.numel())
    squeezed = B.ndim == 1
    if squeezed:
        B = B.unsqueeze(1)
    if nrhs is None:
        nrhs = B.shape[1]
    if B.shape[0] != n:
        raise ValueError(f"B has {B.shape[0]} rows but n={n}")
    B_f = B.t().contiguous()
    dpftrs_raw(_get_handle(), _op(transr), _fill(uplo), n, nrhs, C, B_f, n)
    B.copy_(B_f.t())
    if squeezed:
        B.squeeze_(1)


def dpftri(C: torch.Tensor, *, n: int = None, transr: str = "T", uplo: str = "U") -> None:
    """Overwrite the float64 RFP factor C with the inverse matrix."""
    _get_handle, _fill, _, _n_from_rfp, _, _op, _, _ = _pkg()
    _validate64(C, "C")
    if n is None:
        n = _n_from_rfp(C.numel())
    dpftri_raw(_get_handle(), _op(transr), _fill(uplo), n, C)


def dstrttf(A: torch.Tensor, *, transr: str = "T", uplo: str = "U",
            n: int = None) -> torch.Tensor:
    """Triangle of a square row-major float64 tensor -> new RFP tensor."""
    _get_handle, _fill, _, _, _, _op, _, _ = _pkg()
    _validate64(A, "A")
    if A.ndim != 2 or A.shape[0] != A.shape[1]:
        raise ValueError(f"A must be a square 2-D tensor, got shape {A.shape}")
    if n is None:
        n = A.shape[0]
    arf = torch.empty(n * (n + 1) // 2, dtype=torch.float64, device=A.device)
    dstrttf_raw(_get_handle(), _op(transr), _fill(uplo), n, A, n, arf)
    return arf


def dstfttr(arf: torch.Tensor, *, transr: str = "T", uplo: str = "U",
            n: int = None) -> torch.Tensor:
    """float64 RFP tensor -> new (n, n) tensor with the uplo triangle filled."""
    _get_handle, _fill, _, _n_from_rfp, _, _op, _, _ = _pkg()
    _validate64(arf, "arf")
    if n is None:
        n = _n_from_rfp(arf.numel())
    A = torch.zeros(n, n, dtype=torch.float64, device=arf.device)
    dstfttr_raw(_get_handle(), _op(transr), _fill(uplo), n, arf, A, n)
    return A


def dsfr2k(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor, *, alpha: float = 1.0,
           beta: float = 0.0, transr: str = "T", uplo: str = "U", trans: str = "T",
           n: int = None, k: int = None, lda: int = None, ldb: int = None) -> None:
    """C := alpha*(op(A)op(B)^T + op(B)op(A)^T) + beta*C in RFP, float64."""
    _get_handle, _fill, _, _n_from_rfp, _, _op, _, _ = _pkg()
    if n is None:
        n = _n_from_rfp(C.numel())
    tu = trans.upper()
    if k is None:
        k = A.shape[1] if tu == "T" else A.shape[0]
    if lda is None:
        lda = A.shape[1] if tu == "T" else A.shape[0]
    if ldb is None:
        ldb = B.shape[1] if tu == "T" else B.shape[0]
    dsfr2k_raw(_get_handle(), _op(transr), _fill(uplo), _op(trans), n, k, alpha, A, lda, B,
               ldb, beta, C)


def dlansf(C: torch.Tensor, norm: str = "1", *, transr: str = "T", uplo: str = "U",
           n: int = None) -> float:
    """'M' / '1' / 'F' norm of the symmetric float64 RFP matrix C."""
    _get_handle, _fill, _, _n_from_rfp, _norm, _op, _, _ = _pkg()
    _validate64(C, "C")
    if n is None:
        n = _n_from_rfp(C.numel())
    return dlansf_raw(_get_handle(), _norm(norm), _op(transr), _fill(uplo), n, C)


def dpfcon(C: torch.Tensor, anorm: float, *, transr: str = "T", uplo: str = "U",
           n: int = None) -> float:
    """Reciprocal 1-norm condition estimate from the float64 factor C."""
    _get_handle, _fill, _, _n_from_rfp, _, _op, _, _ = _pkg()
    _validate64(C, "C")
    if n is None:
        n = _n_from_rfp(C.numel())
    return dpfcon_raw(_get_handle(), _op(transr), _fill(uplo), n, C, anorm)


def dpftrf_rcond(C: torch.Tensor, *, transr: str = "T", uplo: str = "U", n: int = None,
                 check: bool = True) -> float:
    """dlansf('1') + in-place dpftrf + dpfcon."""
    _get_handle, _fill, _, _n_from_rfp, _, _op, _, _ = _pkg()
    _validate64(C, "C")
    if n is None:
        n = _n_from_rfp(C.numel())
    h = _get_handle()
    anorm = dlansf_raw(h, 1, _op(transr), _fill(uplo), n, C)
    info = dpftrf_raw(h, _op(transr), _fill(uplo), n, C)
    if check and info != 0:
        raise torch.linalg.LinAlgError(
            f"dpftrf_rcond: matrix is not positive definite "
            f"(leading minor of order {info} is not positive definite)")
    if info != 0 or anorm == 0.0:
        return 0.0
    return dpfcon_raw(h, _op(transr), _fill(uplo), n, C, anorm)


def dsfmv(arf: torch.Tensor, x: torch.Tensor, y: torch.Tensor = None, *, alpha: float = 1.0,
          beta: float = 0.0, transr: str = "T", uplo: str = "U", n: int = None) -> torch.Tensor:
    """y := alpha*A*x + beta*y (float64); returns y."""
    _get_handle, _fill, _, _n_from_rfp, _, _op, _, _ = _pkg()
    _validate64(arf, "arf")
    _validate64(x, "x")
    if n is None:
        n = _n_from_rfp(arf.numel())
    if y is None:
        y = torch.zeros(n, dtype=torch.float64, device=arf.device)
    if x.numel() != n:
        raise ValueError(f"x has {x.numel()} elements but n={n}")
    if y.numel() != n:
        raise ValueError(f"y has {y.numel()} elements but n={n}")
    dsfmv_raw(_get_handle(), _op(transr), _fill(uplo), n, alpha, arf, x, 1, beta, y, 1)
    return y


def dsfmm(arf: torch.Tensor, B: torch.Tensor, C: torch.Tensor = None, *, alpha: float = 1.0,
          beta: float = 0.0, transr: str = "T", uplo: str = "U", side: str = "L",
          n_A: int = None) -> torch.Tensor:
    """side='L': C := alpha*A*B + beta*C; side='R': C := alpha*B*A + beta*C
    (float64; B, C storage handed to the column-major kernel with ld m)."""
    _get_handle, _fill, _, _n_from_rfp, _, _op, _, _side = _pkg()
    _validate64(arf, "arf")
    _validate64(B, "B")
    if B.ndim != 2:
        raise ValueError(f"B must be a 2-D tensor, got shape {B.shape}")
    m, n = B.shape[0], B.shape[1]
    if n_A is None:
        n_A = _n_from_rfp(arf.numel())
    su = side.upper()
    if su == "L" and n_A != m:
        raise ValueError(f"side='L': A is {n_A}x{n_A} but B has {m} rows")
    if su == "R" and n_A != n:
        raise ValueError(f"side='R': A is {n_A}x{n_A} but B has {n} cols")
    if C is None:
        C = torch.zeros(m, n, dtype=torch.float64, device=arf.device)
    _validate64(C, "C")
    if C.shape != (m, n):
        raise ValueError(f"C must be {m}x{n}, got {tuple(C.shape)}")
    dsfmm_raw(_get_handle(), _op(transr), _fill(uplo), _side(side), m, n, alpha, arf, B, m,
              beta, C, m)
    return C


def dsfr(arf: torch.Tensor, x: torch.Tensor, *, alpha: float = 1.0, transr: str = "T",
         uplo: str = "U", n: int = None) -> None:
    """In-place arf := alpha*x*x^T + arf (float64)."""
    _get_handle, _fill, _, _n_from_rfp, _, _op, _, _ = _pkg()
    _validate64(arf, "arf")
    _validate64(x, "x")
    if n is None:
        n = _n_from_rfp(arf.numel())
    if x.numel() != n:
        raise ValueError(f"x must have {n} elements, got {x.numel()}")
    dsfr_raw(_get_handle(), _op(transr), _fill(uplo), n, alpha, x, 1, arf)


def dsfr2(arf: torch.Tensor, x: torch.Tensor, y: torch.Tensor, *, alpha: float = 1.0,
          transr: str = "T", uplo: str = "U", n: int = None) -> None:
    """In-place arf := alpha*(x*y^T + y*x^T) + arf (float64)."""
    _get_handle, _fill, _, _n_from_rfp, _, _op, _, _ = _pkg()
    for t, nm in ((arf, "arf"), (x, "x"), (y, "y")):
        _validate64(t, nm)
    if n is None:
        n = _n_from_rfp(arf.numel())
    if x.numel() != n:
        raise ValueError(f"x must have {n} elements, got {x.numel()}")
    if y.numel() != n:
        raise ValueError(f"y must have {n} elements, got {y.numel()}")
    dsfr2_raw(_get_handle(), _op(transr), _fill(uplo), n, alpha, x, 1, y, 1, arf)


__all__ = [name for name in dir() if name.startswith("d") and not name.startswith("_")]
