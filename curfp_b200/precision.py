"""Precision form: split-BF16 tensor-core contractions and refined solves.

Same call shapes as the drop-in functions, plus ``math``:

* ``math="bf16x3"`` (default here): the large SYRK / GEMM updates of ssfrk and
  of the blocked Cholesky run on the sm_100a tensor cores (tcgen05) with every
  FP32 operand split into three BF16 terms and six BF16 products accumulated in
  FP32; diagonal Cholesky tiles, triangular inverses and small updates stay
  FP32.
* ``math="fp32"``: identical to the drop-in functions.

``spftrs_refined`` wraps the solve in iterative refinement whose residual
b - A x is accumulated in FP64 from the original matrix (the only FP64 step).
"""
from __future__ import annotations

import ctypes

import torch

from . import _get_handle, _n_from_rfp, _op, _fill, _ptr, _validate
from ._lib import check

MATH = {"fp32": 0, "bf16x3": 1}


def _math(m: str) -> int:
    try:
        return MATH[m]
    except KeyError:
        raise ValueError(f"math must be one of {sorted(MATH)}, got {m!r}")


def ssfrk(A: torch.Tensor, C: torch.Tensor, *, alpha: float = 1.0, beta: float = 0.0,
          transr: str = "T", uplo: str = "U", trans: str = "T", n: int = None,
          k: int = None, lda: int = None, math: str = "bf16x3") -> None:
    """C := alpha*op(A)op(A)^T + beta*C in RFP (see curfp_b200.ssfrk)."""
    _validate(A, "A")
    _validate(C, "C")
    if n is None:
        n = _n_from_rfp(C.numel())
    tu = trans.upper()
    if k is None:
        k = A.shape[1] if tu == "T" else A.shape[0]
    if lda is None:
        lda = A.shape[1] if tu == "T" else A.shape[0]
    h = _get_handle()
    a, b = ctypes.c_float(alpha), ctypes.c_float(beta)
    check(h._lib.curfpSsfrkEx(h.ptr, _op(transr), _fill(uplo), _op(trans), n, k,
                              ctypes.byref(a), _ptr(A), lda, ctypes.byref(b), _ptr(C),
                              _math(math)))


def spftrf(C: torch.Tensor, *, n: int = None, transr: str = "T", uplo: str = "U",
           check: bool = True, math: str = "bf16x3") -> int:
    """In-place RFP Cholesky with split-BF16 tensor-core updates."""
    _validate(C, "C")
    if n is None:
        n = _n_from_rfp(C.numel())
    h = _get_handle()
    info = ctypes.c_int(0)
    from ._lib import check as _check
    _check(h._lib.curfpSpftrfEx(h.ptr, _op(transr), _fill(uplo), n, _ptr(C),
                                ctypes.byref(info), _math(math)))
    if check and info.value != 0:
        raise torch.linalg.LinAlgError(
            f"spftrf: matrix is not positive definite "
            f"(leading minor of order {info.value} is not positive definite)")
    return info.value


def spftrf_from_host(C_host: torch.Tensor, C: torch.Tensor, C_orig: torch.Tensor = None, *,
                     n: int = None, transr: str = "T", uplo: str = "U", check: bool = True,
                     math: str = "bf16x3") -> int:
    """Copy the host RFP array C_host (CPU float32, contiguous; pinned for the
    copy to overlap) to the CUDA array C and factor it in place
    (curfpSpftrfFromHost); C_orig, if given, receives the unfactored matrix.
    For transr = T the copy of the array's second part overlaps the
    factorization of the first diagonal block."""
    if C_host.device.type != "cpu" or C_host.dtype != torch.float32 or not C_host.is_contiguous():
        raise ValueError("C_host must be a contiguous float32 CPU tensor")
    _validate(C, "C")
    if C_orig is not None:
        _validate(C_orig, "C_orig")
        if C_orig.numel() != C.numel():
            raise ValueError("C_orig must have as many elements as C")
    if C_host.numel() != C.numel():
        raise ValueError("C_host must have as many elements as C")
    if n is None:
        n = _n_from_rfp(C.numel())
    h = _get_handle()
    info = ctypes.c_int(0)
    from ._lib import check as _check
    _check(h._lib.curfpSpftrfFromHost(h.ptr, _op(transr), _fill(uplo), n,
                                      ctypes.c_void_p(C_host.data_ptr()), _ptr(C),
                                      _ptr(C_orig) if C_orig is not None else None,
                                      ctypes.byref(info), _math(math)))
    if check and info.value != 0:
        raise torch.linalg.LinAlgError(
            f"spftrf: matrix is not positive definite "
            f"(leading minor of order {info.value} is not positive definite)")
    return info.value


def spftrs_refined(A: torch.Tensor, F: torch.Tensor, B: torch.Tensor, *, n: int = None,
                   nrhs: int = None, transr: str = "T", uplo: str = "U",
                   max_iter: int = 3) -> int:
    """Solve A X = B (B (n, nrhs) or (n,), in place) with the factor F of A and
    FP64-residual iterative refinement against A; returns corrections applied."""
    _validate(A, "A")
    _validate(F, "F")
    _validate(B, "B")
    if n is None:
        n = _n_from_rfp(F.numel())
    squeezed = B.ndim == 1
    if squeezed:
        B = B.unsqueeze(1)
    if nrhs is None:
        nrhs = B.shape[1]
    if B.shape[0] != n:
        raise ValueError(f"B has {B.shape[0]} rows but n={n}")
    B_f = B.t().contiguous()
    h = _get_handle()
    iters = ctypes.c_int(0)
    check(h._lib.curfpSpftrsRefine(h.ptr, _op(transr), _fill(uplo), n, nrhs, _ptr(A),
                                   _ptr(F), _ptr(B_f), n, max_iter, ctypes.byref(iters)))
    B.copy_(B_f.t())
    if squeezed:
        B.squeeze_(1)
    return iters.value


def ssfmm_acc64(A: torch.Tensor, X: torch.Tensor, Y: torch.Tensor = None, *,
                alpha: float = 1.0, beta: float = 0.0, transr: str = "T",
                uplo: str = "U", n: int = None) -> torch.Tensor:
    """Y := alpha*A@X + beta*Y for symmetric A in RFP, X/Y (n, nrhs); FP64 sums."""
    _validate(A, "A")
    _validate(X, "X")
    if n is None:
        n = _n_from_rfp(A.numel())
    X2 = X.unsqueeze(1) if X.ndim == 1 else X
    nrhs = X2.shape[1]
    Xf = X2.t().contiguous()
    if Y is None:
        Yf = torch.zeros_like(Xf)
        beta = 0.0
    else:
        _validate(Y, "Y")
        Yf = (Y.unsqueeze(1) if Y.ndim == 1 else Y).t().contiguous()
    h = _get_handle()
    a, b = ctypes.c_float(alpha), ctypes.c_float(beta)
    check(h._lib.curfpSsfmmAcc64(h.ptr, _op(transr), _fill(uplo), n, nrhs, ctypes.byref(a),
                                 _ptr(A), _ptr(Xf), n, ctypes.byref(b), _ptr(Yf), n))
    out = Yf.t()
    if Y is not None:
        Y.copy_(out.reshape(Y.shape))
        return Y
    return out.reshape(X.shape).contiguous()


def launch_count() -> int:
    """Kernels launched through the current device's handle so far."""
    h = _get_handle()
    c = ctypes.c_longlong(0)
    check(h._lib.curfpGetKernelLaunchCount(h.ptr, ctypes.byref(c)))
    return c.value


def release_workspace() -> None:
    """Free the current device handle's workspaces and trim the device pool
    (they grow again on demand)."""
    h = _get_handle()
    check(h._lib.curfpReleaseWorkspace(h.ptr))


def diag_wait_timeout() -> tuple:
    """Self-test of the kernels' bounded waits (~2 s): a wavefront solve whose
    first block row never runs; returns (status, error code), which is
    (CURFP_STATUS_EXECUTION_FAILED, 5) when the waits give up as designed."""
    h = _get_handle()
    code = ctypes.c_int(0)
    st = h._lib.curfpDiagWaitTimeout(h.ptr, ctypes.byref(code))
    return int(st), code.value


KERNEL_CLASSES = ["sgemm", "tc_gemm", "tc_stage", "potrf_tile", "trtri", "lauum",
                  "pack", "diag", "symm_acc64", "trsv_wave", "norm"]


def profile_enable(on: bool = True) -> None:
    """Start (clear) or stop per-kernel-class event timing on this device's handle."""
    h = _get_handle()
    check(h._lib.curfpProfileEnable(h.ptr, 1 if on else 0))


def profile_records() -> list:
    """Every record since profile_enable: dicts with class, ms, flops, bytes
    and (contractions, solves) m, n, k, tiles."""
    import numpy as np
    h = _get_handle()
    n = ctypes.c_longlong(0)
    check(h._lib.curfpProfileRecords(h.ptr, 0, ctypes.byref(n), None))
    buf = np.zeros((max(n.value, 1), 8), np.float64)
    check(h._lib.curfpProfileRecords(h.ptr, n.value, ctypes.byref(n),
                                     buf.ctypes.data_as(ctypes.c_void_p)))
    keys = ("ms", "flops", "bytes", "m", "n", "k", "tiles")
    return [dict(cls=KERNEL_CLASSES[int(r[0])], **{k_: float(v) for k_, v in zip(keys, r[1:])})
            for r in buf[:n.value]]


def profile_read() -> dict:
    """{class: {ms, flops, bytes, launches}} for the records since profile_enable."""
    h = _get_handle()
    out = {}
    for i, name in enumerate(KERNEL_CLASSES):
        ms, fl, by = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        n = ctypes.c_longlong()
        check(h._lib.curfpProfileRead(h.ptr, i, ctypes.byref(ms), ctypes.byref(fl),
                                      ctypes.byref(by), ctypes.byref(n)))
        if n.value:
            out[name] = {"ms": ms.value, "flops": fl.value, "bytes": by.value,
                         "launches": n.value}
    return out
