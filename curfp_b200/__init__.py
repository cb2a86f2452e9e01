"""curfp_b200 — B200-native RFP (Rectangular Full Packed) rank-k update,
Cholesky, solve and inverse, a drop-in for the ``curfp`` Python API.

Same function names, keyword arguments, defaults, string/int enums, error
types and in-place semantics as the reference package (curfp/__init__.py of
andersx/curfp), on the native library libcurfp_b200.so::

    import curfp_b200 as curfp
    curfp.ssfrk(A, C)                 # C = A @ A.T in RFP (transr='T', uplo='U')
    curfp.add_to_diagonal(C, 1.0)
    curfp.spftrf(C)                   # in-place Cholesky
    curfp.spftrs(C, B)                # solve, B (n, nrhs) overwritten
"""
from __future__ import annotations

import ctypes
import math

import torch

from . import _lib
from ._lib import CurfpError, check

__all__ = [
    "OP_N", "OP_T", "FILL_LOWER", "FILL_UPPER", "Handle", "set_stream",
    "rfp_diag_indices", "add_to_diagonal", "ssfrk", "ssfrk_raw", "spftrf",
    "spftrf_raw", "spftrs", "spftrs_raw", "spftri", "spftri_raw", "strttf",
    "strttf_raw", "stfttr", "stfttr_raw", "ssfr2k", "ssfr2k_raw", "CurfpError",
    "NORM_MAX", "NORM_ONE", "NORM_FRO", "slansf", "slansf_raw", "spfcon", "spfcon_raw",
    "spftrf_rcond", "SIDE_LEFT", "SIDE_RIGHT", "ssfmm", "ssfmm_raw", "ssfmv", "ssfmv_raw",
    "ssfr", "ssfr_raw", "ssfr2", "ssfr2_raw", "set_math_mode", "get_math_mode",
]

# Enum values of include/curfp.h (reference curfp/_ext.cpp:869-877).
OP_N, OP_T = 0, 1
FILL_LOWER, FILL_UPPER = 0, 1
NORM_MAX, NORM_ONE, NORM_FRO = 0, 1, 2
SIDE_LEFT, SIDE_RIGHT = 0, 1


class Handle:
    """Library handle (stream + device state), reference curfp/_ext.cpp:30-44
    and curfp/__init__.py:302-317.  Usable as a context manager."""

    def __init__(self):
        lib = _lib.load()
        h = ctypes.c_void_p()
        check(lib.curfpCreate(ctypes.byref(h)))
        self._h = h
        self._lib = lib

    @property
    def ptr(self) -> ctypes.c_void_p:
        return self._h

    def set_stream_ptr(self, ptr: int) -> None:
        check(self._lib.curfpSetStream(self._h, ctypes.c_void_p(int(ptr))))

    def set_stream(self, stream: torch.cuda.Stream) -> None:
        self.set_stream_ptr(stream.cuda_stream)

    def get_stream_ptr(self) -> int:
        s = ctypes.c_void_p()
        check(self._lib.curfpGetStream(self._h, ctypes.byref(s)))
        return int(s.value or 0)

    def set_math_mode(self, mode: str) -> None:
        """Contraction arithmetic of the FP32 routines on this handle:
        "bf16x3" (default: split-BF16 tensor-core contractions) or "fp32"
        (FP32 FMA on the SIMT cores)."""
        check(self._lib.curfpSetMathMode(self._h, _MATH_MODES[_math_key(mode)]))

    def get_math_mode(self) -> str:
        m = ctypes.c_int(0)
        check(self._lib.curfpGetMathMode(self._h, ctypes.byref(m)))
        return {v: k for k, v in _MATH_MODES.items()}[m.value]

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.curfpDestroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


_MATH_MODES = {"fp32": 0, "bf16x3": 1}


def _math_key(mode: str) -> str:
    if mode not in _MATH_MODES:
        raise ValueError(f"math mode must be one of {sorted(_MATH_MODES)}, got {mode!r}")
    return mode


_handles: dict = {}


def _get_handle() -> Handle:
    dev = torch.cuda.current_device()
    if dev not in _handles:
        _handles[dev] = Handle()
    return _handles[dev]


def set_math_mode(mode: str) -> None:
    """Contraction arithmetic of the FP32 routines on the current device's
    handle: "bf16x3" (the default, split-BF16 tensor cores) or "fp32" (SIMT
    FP32 FMA).  No counterpart in the reference."""
    _get_handle().set_math_mode(mode)


def get_math_mode() -> str:
    return _get_handle().get_math_mode()


def set_stream(stream) -> None:
    """Bind curfp work on the current device to ``stream`` (None: default
    stream), reference curfp/__init__.py:98-106."""
    h = _get_handle()
    h.set_stream_ptr(0 if stream is None else stream.cuda_stream)


_OP_MAP = {"N": OP_N, "T": OP_T}
_FILL_MAP = {"L": FILL_LOWER, "U": FILL_UPPER}


def _op(s: str) -> int:
    try:
        return _OP_MAP[s.upper()]
    except KeyError:
        raise ValueError(f"transr/trans must be 'N' or 'T', got {s!r}")


def _fill(s: str) -> int:
    try:
        return _FILL_MAP[s.upper()]
    except KeyError:
        raise ValueError(f"uplo must be 'L' or 'U', got {s!r}")


# norm strings of reference curfp/__init__.py:114-123
_NORM_MAP = {"M": NORM_MAX, "MAX": NORM_MAX, "1": NORM_ONE, "O": NORM_ONE, "I": NORM_ONE,
             "F": NORM_FRO, "E": NORM_FRO, "FRO": NORM_FRO}


def _norm(s: str) -> int:
    try:
        return _NORM_MAP[s.upper()]
    except KeyError:
        raise ValueError(f"norm must be 'M'/'1'/'F' (or 'O'/'I'/'E'), got {s!r}")


_SIDE_MAP = {"L": SIDE_LEFT, "R": SIDE_RIGHT}


def _side(s: str) -> int:
    try:
        return _SIDE_MAP[s.upper()]
    except KeyError:
        raise ValueError(f"side must be 'L' or 'R', got {s!r}")


def _n_from_rfp(numel: int) -> int:
    n = int((-1.0 + math.sqrt(1.0 + 8.0 * numel)) / 2.0)
    if n * (n + 1) // 2 != numel:
        raise ValueError(
            f"Tensor has {numel} elements which is not a valid RFP size n*(n+1)//2")
    return n


def _validate(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if t.dtype != torch.float32:
        raise ValueError(f"{name} must be float32 (got {t.dtype})")


def _ptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _hp(h) -> ctypes.c_void_p:
    return h.ptr if isinstance(h, Handle) else h


# ---------------------------------------------------------------------------
# Diagonal utilities (reference curfp/__init__.py:194-296), as kernels.
# ---------------------------------------------------------------------------
def rfp_diag_indices(n: int, transr: str = "T", uplo: str = "U",
                     device=None) -> torch.Tensor:
    """int64 tensor of the flat RFP offsets of the n diagonal elements."""
    if device is None:
        device = torch.cuda.current_device()
    idx = torch.empty(n, dtype=torch.int64, device=device)
    with torch.cuda.device(idx.device):
        h = _get_handle()
        check(h._lib.curfpRfpDiagIndices(h.ptr, _op(transr), _fill(uplo), n,
                                         _ptr(idx)))
    return idx


def add_to_diagonal(C: torch.Tensor, value: float, transr: str = "T",
                    uplo: str = "U", n: int = None) -> None:
    """M := M + value*I for the symmetric matrix held in RFP tensor C."""
    if not C.is_cuda:
        raise ValueError("C must be a CUDA tensor")
    if not C.is_contiguous():
        raise ValueError("C must be contiguous")
    if C.dtype not in (torch.float32, torch.float64):
        raise ValueError(f"C must be float32 or float64 (got {C.dtype})")
    if n is None:
        n = _n_from_rfp(C.numel())
    with torch.cuda.device(C.device):
        h = _get_handle()
        if C.dtype == torch.float32:
            check(h._lib.curfpSaddToDiagonal(h.ptr, _op(transr), _fill(uplo), n,
                                             float(value), _ptr(C)))
        else:
            check(h._lib.curfpDaddToDiagonal(h.ptr, _op(transr), _fill(uplo), n,
                                             float(value), _ptr(C)))


# ---------------------------------------------------------------------------
# Raw API (reference curfp/__init__.py:323-404, 689-716, 1164-1197)
# ---------------------------------------------------------------------------
def ssfrk_raw(handle, transr: int, uplo: int, trans: int, n: int, k: int,
              alpha: float, A: torch.Tensor, lda: int, beta: float,
              C: torch.Tensor) -> None:
    if A is not None:
        _validate(A, "A")
    _validate(C, "C")
    a, b = ctypes.c_float(alpha), ctypes.c_float(beta)
    check(_lib.load().curfpSsfrk(_hp(handle), transr, uplo, trans, n, k,
                                 ctypes.byref(a), _ptr(A), lda, ctypes.byref(b),
                                 _ptr(C)))


def spftrf_raw(handle, transr: int, uplo: int, n: int, A: torch.Tensor) -> int:
    _validate(A, "A")
    info = ctypes.c_int(0)
    check(_lib.load().curfpSpftrf(_hp(handle), transr, uplo, n, _ptr(A),
                                  ctypes.byref(info)))
    return info.value


def spftrs_raw(handle, transr: int, uplo: int, n: int, nrhs: int,
               A: torch.Tensor, B: torch.Tensor, ldb: int) -> None:
    _validate(A, "A")
    _validate(B, "B")
    check(_lib.load().curfpSpftrs(_hp(handle), transr, uplo, n, nrhs, _ptr(A),
                                  _ptr(B), ldb))


def spftri_raw(handle, transr: int, uplo: int, n: int, A: torch.Tensor) -> None:
    _validate(A, "A")
    check(_lib.load().curfpSpftri(_hp(handle), transr, uplo, n, _ptr(A)))


def strttf_raw(handle, transr: int, uplo: int, n: int, A: torch.Tensor,
               lda: int, arf: torch.Tensor) -> None:
    _validate(A, "A")
    _validate(arf, "arf")
    check(_lib.load().curfpSstrttf(_hp(handle), transr, uplo, n, _ptr(A), lda,
                                   _ptr(arf)))


def stfttr_raw(handle, transr: int, uplo: int, n: int, arf: torch.Tensor,
               A: torch.Tensor, lda: int) -> None:
    _validate(arf, "arf")
    _validate(A, "A")
    check(_lib.load().curfpSstfttr(_hp(handle), transr, uplo, n, _ptr(arf),
                                   _ptr(A), lda))


def ssfr2k_raw(handle, transr: int, uplo: int, trans: int, n: int, k: int,
               alpha: float, A: torch.Tensor, lda: int, B: torch.Tensor,
               ldb: int, beta: float, C: torch.Tensor) -> None:
    _validate(A, "A")
    _validate(B, "B")
    _validate(C, "C")
    a, b = ctypes.c_float(alpha), ctypes.c_float(beta)
    check(_lib.load().curfpSsfr2k(_hp(handle), transr, uplo, trans, n, k,
                                  ctypes.byref(a), _ptr(A), lda, _ptr(B), ldb,
                                  ctypes.byref(b), _ptr(C)))


# ---------------------------------------------------------------------------
# High-level API (reference curfp/__init__.py:410-565, 661-781, 1100-1161)
# ---------------------------------------------------------------------------
def ssfrk(A: torch.Tensor, C: torch.Tensor, *, alpha: float = 1.0,
          beta: float = 0.0, transr: str = "T", uplo: str = "U",
          trans: str = "T", n: int = None, k: int = None,
          lda: int = None) -> None:
    """C := alpha*A@A.T + beta*C (trans='T', A row-major n x k) or
    alpha*A.T@A + beta*C (trans='N', A column-major n x k), C in RFP."""
    _validate(A, "A")
    _validate(C, "C")
    if n is None:
        n = _n_from_rfp(C.numel())
    tu = trans.upper()
    if k is None:
        k = A.shape[1] if tu == "T" else A.shape[0]
    if lda is None:
        lda = A.shape[1] if tu == "T" else A.shape[0]
    ssfrk_raw(_get_handle(), _op(transr), _fill(uplo), _op(trans), n, k,
              alpha, A, lda, beta, C)


def spftrf(C: torch.Tensor, *, n: int = None, transr: str = "T",
           uplo: str = "U", check: bool = True) -> int:
    """In-place RFP Cholesky; returns info (raises LinAlgError if check)."""
    _validate(C, "C")
    if n is None:
        n = _n_from_rfp(C.numel())
    info = spftrf_raw(_get_handle(), _op(transr), _fill(uplo), n, C)
    if check and info != 0:
        raise torch.linalg.LinAlgError(
            f"spftrf: matrix is not positive definite "
            f"(leading minor of order {info} is not positive definite)")
    return info


def spftrs(C: torch.Tensor, B: torch.Tensor, *, n: int = None,
           nrhs: int = None, transr: str = "T", uplo: str = "U") -> None:
    """Solve A X = B with the RFP factor C; B (n, nrhs) or (n,) in place."""
    _validate(C, "C")
    _validate(B, "B")
    if n is None:
        n = _n_from_rfp(C.numel())
    squeezed = B.ndim == 1
    if squeezed:
        B = B.unsqueeze(1)
    if nrhs is None:
        nrhs = B.shape[1]
    if B.shape[0] != n:
        raise ValueError(f"B has {B.shape[0]} rows but n={n}")
    B_f = B.t().contiguous()  # (nrhs, n) C-order == column-major n x nrhs
    spftrs_raw(_get_handle(), _op(transr), _fill(uplo), n, nrhs, C, B_f, n)
    B.copy_(B_f.t())
    if squeezed:
        B.squeeze_(1)


def spftri(C: torch.Tensor, *, n: int = None, transr: str = "T",
           uplo: str = "U") -> None:
    """Overwrite the RFP Cholesky factor C with the inverse matrix."""
    _validate(C, "C")
    if n is None:
        n = _n_from_rfp(C.numel())
    spftri_raw(_get_handle(), _op(transr), _fill(uplo), n, C)


def strttf(A: torch.Tensor, *, transr: str = "T", uplo: str = "U",
           n: int = None) -> torch.Tensor:
    """Triangle of a square row-major tensor -> new RFP tensor."""
    _validate(A, "A")
    if A.ndim != 2 or A.shape[0] != A.shape[1]:
        raise ValueError(f"A must be a square 2-D tensor, got shape {A.shape}")
    if n is None:
        n = A.shape[0]
    arf = torch.empty(n * (n + 1) // 2, dtype=torch.float32, device=A.device)
    strttf_raw(_get_handle(), _op(transr), _fill(uplo), n, A, n, arf)
    return arf


def stfttr(arf: torch.Tensor, *, transr: str = "T", uplo: str = "U",
           n: int = None) -> torch.Tensor:
    """RFP tensor -> new (n, n) tensor with the uplo triangle filled."""
    _validate(arf, "arf")
    if n is None:
        n = _n_from_rfp(arf.numel())
    A = torch.zeros(n, n, dtype=torch.float32, device=arf.device)
    stfttr_raw(_get_handle(), _op(transr), _fill(uplo), n, arf, A, n)
    return A


def ssfr2k(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor, *,
           alpha: float = 1.0, beta: float = 0.0, transr: str = "T",
           uplo: str = "U", trans: str = "T", n: int = None, k: int = None,
           lda: int = None, ldb: int = None) -> None:
    """C := alpha*(op(A)op(B)^T + op(B)op(A)^T) + beta*C in RFP."""
    _validate(A, "A")
    _validate(B, "B")
    _validate(C, "C")
    if n is None:
        n = _n_from_rfp(C.numel())
    tu = trans.upper()
    if k is None:
        k = A.shape[1] if tu == "T" else A.shape[0]
    if lda is None:
        lda = A.shape[1] if tu == "T" else A.shape[0]
    if ldb is None:
        ldb = B.shape[1] if tu == "T" else B.shape[0]
    ssfr2k_raw(_get_handle(), _op(transr), _fill(uplo), _op(trans), n, k,
               alpha, A, lda, B, ldb, beta, C)


# ---------------------------------------------------------------------------
# Norms and condition estimate (reference curfp/__init__.py:784-960)
# ---------------------------------------------------------------------------

def slansf_raw(handle, norm: int, transr: int, uplo: int, n: int, C: torch.Tensor) -> float:
    """Norm (NORM_MAX / NORM_ONE / NORM_FRO) of the symmetric RFP matrix C."""
    _validate(C, "C")
    out = ctypes.c_float(0.0)
    check(_lib.load().curfpSlansf(_hp(handle), norm, transr, uplo, n, _ptr(C),
                                  ctypes.byref(out)))
    return float(out.value)


def slansf(C: torch.Tensor, norm: str = "1", *, transr: str = "T", uplo: str = "U",
           n: int = None) -> float:
    """'M' max |A(i,j)|, '1' / 'O' / 'I' max column sum of |A|, 'F' / 'E'
    Frobenius norm, of the symmetric matrix held in C (RFP, not a factor)."""
    _validate(C, "C")
    if n is None:
        n = _n_from_rfp(C.numel())
    return slansf_raw(_get_handle(), _norm(norm), _op(transr), _fill(uplo), n, C)


def spfcon_raw(handle, transr: int, uplo: int, n: int, C: torch.Tensor, anorm: float) -> float:
    """rcond = 1 / (||A^-1||_1 anorm) from the RFP Cholesky factor C."""
    _validate(C, "C")
    out = ctypes.c_float(0.0)
    check(_lib.load().curfpSpfcon(_hp(handle), transr, uplo, n, _ptr(C), float(anorm),
                                  ctypes.byref(out)))
    return float(out.value)


def spfcon(C: torch.Tensor, anorm: float, *, transr: str = "T", uplo: str = "U",
           n: int = None) -> float:
    """Reciprocal condition number estimate (Hager-Higham 1-norm estimator)
    from the factor C left by spftrf; anorm = slansf(A, '1') of the matrix
    before factorization.  0.0 if anorm == 0."""
    _validate(C, "C")
    if n is None:
        n = _n_from_rfp(C.numel())
    return spfcon_raw(_get_handle(), _op(transr), _fill(uplo), n, C, anorm)


def spftrf_rcond(C: torch.Tensor, *, transr: str = "T", uplo: str = "U", n: int = None,
                 check: bool = True) -> float:
    """slansf('1') + in-place spftrf + spfcon: factor C and return its
    estimated reciprocal condition number (0.0 if not positive definite and
    check=False)."""
    _validate(C, "C")
    if n is None:
        n = _n_from_rfp(C.numel())
    h = _get_handle()
    anorm = slansf_raw(h, NORM_ONE, _op(transr), _fill(uplo), n, C)
    info = spftrf_raw(h, _op(transr), _fill(uplo), n, C)
    if check and info != 0:
        raise torch.linalg.LinAlgError(
            f"spftrf_rcond: matrix is not positive definite "
            f"(leading minor of order {info} is not positive definite)")
    if info != 0 or anorm == 0.0:
        return 0.0
    return spfcon_raw(h, _op(transr), _fill(uplo), n, C, anorm)


# ---------------------------------------------------------------------------
# Symmetric (RFP) times dense (reference curfp/__init__.py:568-650, 1203-1340)
# ---------------------------------------------------------------------------

def ssfmv_raw(handle, transr: int, uplo: int, n: int, alpha: float, arf: torch.Tensor,
              x: torch.Tensor, incx: int, beta: float, y: torch.Tensor, incy: int) -> None:
    """y := alpha*A*x + beta*y in place (BLAS increments)."""
    _validate(arf, "arf")
    _validate(x, "x")
    _validate(y, "y")
    a, b = ctypes.c_float(alpha), ctypes.c_float(beta)
    check(_lib.load().curfpSsfmv(_hp(handle), transr, uplo, n, ctypes.byref(a), _ptr(arf),
                                 _ptr(x), incx, ctypes.byref(b), _ptr(y), incy))


def ssfmv(arf: torch.Tensor, x: torch.Tensor, y: torch.Tensor = None, *, alpha: float = 1.0,
          beta: float = 0.0, transr: str = "T", uplo: str = "U", n: int = None) -> torch.Tensor:
    """y := alpha*A*x + beta*y with A symmetric in RFP; y created (zeros) if
    not given; returns y."""
    _validate(arf, "arf")
    _validate(x, "x")
    if n is None:
        n = _n_from_rfp(arf.numel())
    if y is None:
        y = torch.zeros(n, dtype=torch.float32, device=arf.device)
    _validate(y, "y")
    if x.numel() != n:
        raise ValueError(f"x has {x.numel()} elements but n={n}")
    if y.numel() != n:
        raise ValueError(f"y has {y.numel()} elements but n={n}")
    ssfmv_raw(_get_handle(), _op(transr), _fill(uplo), n, alpha, arf, x, 1, beta, y, 1)
    return y


def ssfmm_raw(handle, transr: int, uplo: int, side: int, m: int, n: int, alpha: float,
              arf: torch.Tensor, B: torch.Tensor, ldb: int, beta: float, C: torch.Tensor,
              ldc: int) -> None:
    """C := alpha*A*B + beta*C (side LEFT) or alpha*B*A + beta*C (RIGHT);
    B, C column-major m x n with leading dimensions ldb, ldc."""
    _validate(arf, "arf")
    _validate(B, "B")
    _validate(C, "C")
    a, b = ctypes.c_float(alpha), ctypes.c_float(beta)
    check(_lib.load().curfpSsfmm(_hp(handle), transr, uplo, side, m, n, ctypes.byref(a),
                                 _ptr(arf), _ptr(B), ldb, ctypes.byref(b), _ptr(C), ldc))


def ssfmm(arf: torch.Tensor, B: torch.Tensor, C: torch.Tensor = None, *, alpha: float = 1.0,
          beta: float = 0.0, transr: str = "T", uplo: str = "U", side: str = "L",
          n_A: int = None) -> torch.Tensor:
    """side='L': C := alpha*A*B + beta*C (A m x m); side='R': C := alpha*B*A
    + beta*C (A n x n), B and C of shape (m, n).  As in the reference, the
    storage of B and C is handed to the column-major kernel with leading
    dimension m; returns C (zeros if not given)."""
    _validate(arf, "arf")
    _validate(B, "B")
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
        C = torch.zeros(m, n, dtype=torch.float32, device=arf.device)
    _validate(C, "C")
    if C.shape != (m, n):
        raise ValueError(f"C must be {m}x{n}, got {tuple(C.shape)}")
    ssfmm_raw(_get_handle(), _op(transr), _fill(uplo), _side(side), m, n, alpha, arf, B, m,
              beta, C, m)
    return C


# ---------------------------------------------------------------------------
# Rank-1 / rank-2 updates (reference curfp/__init__.py:966-1097)
# ---------------------------------------------------------------------------

def ssfr_raw(handle, transr: int, uplo: int, n: int, alpha: float, x: torch.Tensor,
             incx: int, arf: torch.Tensor) -> None:
    """arf := alpha*x*x^T + arf (BLAS increment incx)."""
    _validate(x, "x")
    _validate(arf, "arf")
    a = ctypes.c_float(alpha)
    check(_lib.load().curfpSsfr(_hp(handle), transr, uplo, n, ctypes.byref(a), _ptr(x), incx,
                                _ptr(arf)))


def ssfr(arf: torch.Tensor, x: torch.Tensor, *, alpha: float = 1.0, transr: str = "T",
         uplo: str = "U", n: int = None) -> None:
    """In-place symmetric rank-1 update arf := alpha*x*x^T + arf (RFP)."""
    _validate(arf, "arf")
    _validate(x, "x")
    if n is None:
        n = _n_from_rfp(arf.numel())
    if x.numel() != n:
        raise ValueError(f"x must have {n} elements, got {x.numel()}")
    ssfr_raw(_get_handle(), _op(transr), _fill(uplo), n, alpha, x, 1, arf)


def ssfr2_raw(handle, transr: int, uplo: int, n: int, alpha: float, x: torch.Tensor,
              incx: int, y: torch.Tensor, incy: int, arf: torch.Tensor) -> None:
    """arf := alpha*(x*y^T + y*x^T) + arf (BLAS increments)."""
    _validate(x, "x")
    _validate(y, "y")
    _validate(arf, "arf")
    a = ctypes.c_float(alpha)
    check(_lib.load().curfpSsfr2(_hp(handle), transr, uplo, n, ctypes.byref(a), _ptr(x), incx,
                                 _ptr(y), incy, _ptr(arf)))


def ssfr2(arf: torch.Tensor, x: torch.Tensor, y: torch.Tensor, *, alpha: float = 1.0,
          transr: str = "T", uplo: str = "U", n: int = None) -> None:
    """In-place symmetric rank-2 update arf := alpha*(x*y^T + y*x^T) + arf."""
    _validate(arf, "arf")
    _validate(x, "x")
    _validate(y, "y")
    if n is None:
        n = _n_from_rfp(arf.numel())
    if x.numel() != n:
        raise ValueError(f"x must have {n} elements, got {x.numel()}")
    if y.numel() != n:
        raise ValueError(f"y must have {n} elements, got {y.numel()}")
    ssfr2_raw(_get_handle(), _op(transr), _fill(uplo), n, alpha, x, 1, y, 1, arf)


# FP64 (D-prefix) twins (reference curfp/__init__.py:1347-2090).
from ._double import *  # noqa: E402,F401,F403
from ._double import __all__ as _double_all  # noqa: E402

__all__ += _double_all
