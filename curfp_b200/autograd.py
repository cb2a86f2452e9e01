"""Differentiation form: RFP rank-k update, Cholesky and solve as
``torch.autograd.Function``s with hand-written adjoints (library entry points
curfpSsfrkBackward, curfpSpftrfBackward, curfpSpftrsBackward).

Cotangents of RFP tensors are RFP tensors of the same variant holding the
derivative with respect to each STORED element; an off-diagonal stored element
stands for two entries of the symmetric matrix.  Composed functions therefore
agree with dense autograd on the unpacked matrices (the tests check this
against ``torch.linalg.cholesky`` in FP64).

* ``ssfrk(A, alpha)``: C = alpha A A^T (A row-major n x k).
  Abar = alpha (tril(Cbar) + tril(Cbar)^T) A, alphabar = <Cbar, A A^T>_stored.
* ``add_to_diagonal(C, value)``: C + value I; valuebar = sum of Cbar's diagonal.
* ``cholesky(C)``: L with C = L L^T.  Cbar = packed lower triangle of
  S = L^-T Q L^-1 with Q = sym(tril(L^T Lbar)), diagonal halved.  Only L is
  kept for the backward; its triangular solves are recomputed from L.
* ``solve(L, B)``: X = (L L^T)^-1 B.  Bbar = (L L^T)^-1 Xbar,
  Lbar = -tril(Bbar (L^T X)^T + X (L^T Bbar)^T).
* ``log_diag_sum(L)``: sum_i log L_ii (log-determinant / 2).
* ``nll(X, s, sigma2, y)``: 1/2 y^T C^-1 y + sum log diag(L) with
  C = s X X^T + sigma2 I, the Gaussian-process negative log marginal
  likelihood up to its constant.  Fused (default): one Function whose forward
  solves for alpha = C^-1 y with FP64-residual iterative refinement and whose
  backward (curfpSgpnllBackward) evaluates Cbar = 1/2 (C^-1 - alpha alpha^T)
  through X: Xbar = s (C^-1 X - alpha (alpha^T X)), sbar = <Cbar, X X^T>,
  sigma2bar = tr Cbar, keeping only L, X and alpha.  ``fused=False`` composes
  the per-op Functions above instead.

``math`` ("fp32" or "bf16x3") selects the contraction arithmetic of the
factorization and of the Cholesky adjoint's triangular solves.

Every library call goes through the torch extension (torch.ops.curfp_b200.*,
curfp_b200/csrc_torch/torch_ops.cpp), on torch's current stream: the autograd
engine runs a backward on the stream of its forward.
"""
from __future__ import annotations

import torch

from . import _fill, _n_from_rfp, _op, rfp_diag_indices
from ._torch_ops import ops
from .precision import _math

__all__ = ["ssfrk", "add_to_diagonal", "cholesky", "solve", "log_diag_sum", "nll"]


def _check_rfp(t: torch.Tensor, name: str) -> int:
    if not t.is_cuda or t.dtype != torch.float32 or t.ndim != 1:
        raise ValueError(f"{name} must be a 1-D float32 CUDA tensor (RFP array)")
    return _n_from_rfp(t.numel())


_diag_cache: dict = {}


def _diag_idx(n: int, transr: str, uplo: str, device) -> torch.Tensor:
    key = (n, transr.upper(), uplo.upper(), str(device))
    idx = _diag_cache.get(key)
    if idx is None:
        idx = _diag_cache[key] = rfp_diag_indices(n, transr, uplo, device=device)
    return idx


def _scalar(v) -> float:
    return float(v.detach()) if torch.is_tensor(v) else float(v)


class _Ssfrk(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A, alpha, transr, uplo, math):
        if not A.is_cuda or A.dtype != torch.float32 or A.ndim != 2:
            raise ValueError("A must be a 2-D float32 CUDA tensor")
        A = A.contiguous()
        n, k = A.shape
        a = _scalar(alpha)
        C = torch.empty(n * (n + 1) // 2, device=A.device, dtype=torch.float32)
        ops().ssfrk(A, C, a, 0.0, _op(transr), _fill(uplo), 1, n, k, max(k, 1), _math(math))
        ctx.save_for_backward(A)
        ctx.alpha, ctx.transr, ctx.uplo = a, transr, uplo
        ctx.alpha_is_tensor = torch.is_tensor(alpha)
        return C

    @staticmethod
    def backward(ctx, Cbar):
        (A,) = ctx.saved_tensors
        need_a, need_alpha = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        if not (need_a or need_alpha):
            return None, None, None, None, None
        Cbar = Cbar.contiguous()
        n, k = A.shape
        G = torch.empty_like(A)
        scale = 1.0 if need_alpha else ctx.alpha
        ops().ssfrk_backward(A, Cbar, G, scale, _op(ctx.transr), _fill(ctx.uplo), 1, n, k,
                             max(k, 1))
        g_alpha = 0.5 * torch.sum(G * A) if need_alpha else None
        g_a = (G * ctx.alpha if need_alpha else G) if need_a else None
        return g_a, g_alpha, None, None, None


class _AddDiag(torch.autograd.Function):
    @staticmethod
    def forward(ctx, C, value, transr, uplo):
        n = _check_rfp(C, "C")
        out = C.contiguous().clone()
        ops().add_to_diagonal(out, _scalar(value), _op(transr), _fill(uplo), n)
        ctx.n, ctx.transr, ctx.uplo = n, transr, uplo
        return out

    @staticmethod
    def backward(ctx, Cbar):
        g_value = None
        if ctx.needs_input_grad[1]:
            idx = _diag_idx(ctx.n, ctx.transr, ctx.uplo, Cbar.device)
            g_value = Cbar.index_select(0, idx).sum()
        return Cbar, g_value, None, None


class _Cholesky(torch.autograd.Function):
    @staticmethod
    def forward(ctx, C, transr, uplo, math):
        n = _check_rfp(C, "C")
        L = C.contiguous().clone()
        info = ops().spftrf(L, _op(transr), _fill(uplo), n, _math(math))
        if info != 0:
            raise torch.linalg.LinAlgError(
                f"cholesky: matrix is not positive definite (leading minor of order "
                f"{info} is not positive definite)")
        ctx.save_for_backward(L)
        ctx.n, ctx.transr, ctx.uplo, ctx.math = n, transr, uplo, math
        return L

    @staticmethod
    def backward(ctx, Lbar):
        (L,) = ctx.saved_tensors
        Lbar = Lbar.contiguous()
        Cbar = torch.empty_like(L)
        ops().spftrf_backward(L, Lbar, Cbar, _op(ctx.transr), _fill(ctx.uplo), ctx.n,
                              _math(ctx.math))
        return Cbar, None, None, None


class _Solve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, L, B, transr, uplo):
        n = _check_rfp(L, "L")
        if not B.is_cuda or B.dtype != torch.float32 or B.ndim not in (1, 2):
            raise ValueError("B must be a float32 CUDA tensor of shape (n,) or (n, nrhs)")
        if B.shape[0] != n:
            raise ValueError(f"B has {B.shape[0]} rows but n={n}")
        vec = B.ndim == 1
        Bm = B.unsqueeze(1) if vec else B
        nrhs = Bm.shape[1]
        # (nrhs, n) row-major == column-major n x nrhs, always a fresh buffer
        # (for nrhs = 1, Bm.t() is already contiguous and would alias B)
        Xf = torch.empty((nrhs, n), device=B.device, dtype=torch.float32).copy_(Bm.t())
        ops().spftrs(L, Xf, _op(transr), _fill(uplo), n, nrhs, n)
        ctx.save_for_backward(L, Xf)
        ctx.n, ctx.transr, ctx.uplo, ctx.vec = n, transr, uplo, vec
        X = Xf.t()
        return X.squeeze(1).clone() if vec else X.contiguous()

    @staticmethod
    def backward(ctx, Xbar):
        L, Xf = ctx.saved_tensors
        n, nrhs = ctx.n, Xf.shape[0]
        Xbm = Xbar.unsqueeze(1) if ctx.vec else Xbar
        # column-major n x nrhs, solved in place: never the incoming gradient
        Bbf = torch.empty((nrhs, n), device=Xbar.device, dtype=torch.float32).copy_(Xbm.t())
        need_l = ctx.needs_input_grad[0]
        Lbar = torch.empty_like(L) if need_l else None
        ops().spftrs_backward(L, Xf, Bbf, Lbar if need_l else L.new_empty(0),
                              _op(ctx.transr), _fill(ctx.uplo), n, nrhs)
        Bbar = None
        if ctx.needs_input_grad[1]:
            Bbar = Bbf.t()
            Bbar = Bbar.squeeze(1).clone() if ctx.vec else Bbar.contiguous()
        return Lbar, Bbar, None, None


class _GpNll(torch.autograd.Function):
    @staticmethod
    def forward(ctx, X, s, sigma2, y, transr, uplo, math, refine):
        if not X.is_cuda or X.dtype != torch.float32 or X.ndim != 2:
            raise ValueError("X must be a 2-D float32 CUDA tensor")
        if y.dtype != torch.float32 or y.shape != (X.shape[0],):
            raise ValueError("y must be a float32 tensor of shape (n,)")
        X = X.contiguous()
        n, d = X.shape
        sv, vv = _scalar(s), _scalar(sigma2)
        C = torch.empty(n * (n + 1) // 2, device=X.device, dtype=torch.float32)
        a = y.detach().clone().contiguous()
        o = ops()
        o.ssfrk(X, C, sv, 0.0, _op(transr), _fill(uplo), 1, n, d, max(d, 1), _math(math))
        o.add_to_diagonal(C, vv, _op(transr), _fill(uplo), n)
        L = C.clone()
        info = o.spftrf(L, _op(transr), _fill(uplo), n, _math(math))
        if info != 0:
            raise torch.linalg.LinAlgError(
                f"nll: C is not positive definite (leading minor of order {info})")
        o.spftrs_refine(C, L, a, _op(transr), _fill(uplo), n, 1, n, int(refine))
        del C
        idx = _diag_idx(n, transr, uplo, X.device)
        loss = (0.5 * torch.dot(y.detach().double(), a.double())
                + torch.log(L.index_select(0, idx).double()).sum())
        ctx.save_for_backward(X, L, a)
        ctx.sv, ctx.transr, ctx.uplo, ctx.math = sv, transr, uplo, math
        ctx.s_shape = s.shape if torch.is_tensor(s) else None
        ctx.v_shape = sigma2.shape if torch.is_tensor(sigma2) else None
        return loss.float()

    @staticmethod
    def backward(ctx, g):
        X, L, a = ctx.saved_tensors
        n, d = X.shape
        gx = torch.empty_like(X)
        sums = torch.empty(2, device=X.device, dtype=torch.float64)
        g32 = g.detach().float().contiguous()
        ops().gpnll_backward(L, X, a, g32, gx, sums, ctx.sv, _op(ctx.transr), _fill(ctx.uplo),
                             n, d, _math(ctx.math))
        gs = sums[0].float().reshape(ctx.s_shape) if ctx.needs_input_grad[1] else None
        gv = sums[1].float().reshape(ctx.v_shape) if ctx.needs_input_grad[2] else None
        gy = a * g32 if ctx.needs_input_grad[3] else None
        return (gx if ctx.needs_input_grad[0] else None), gs, gv, gy, None, None, None, None


def ssfrk(A: torch.Tensor, alpha=1.0, *, transr: str = "T", uplo: str = "U",
          math: str = "fp32") -> torch.Tensor:
    """New RFP tensor C = alpha * A @ A.T (A row-major n x k); differentiable
    in A and in alpha (a float or a 0-d tensor)."""
    return _Ssfrk.apply(A, alpha, transr, uplo, math)


def add_to_diagonal(C: torch.Tensor, value, *, transr: str = "T",
                    uplo: str = "U") -> torch.Tensor:
    """New RFP tensor C + value * I; differentiable in C and value."""
    return _AddDiag.apply(C, value, transr, uplo)


def cholesky(C: torch.Tensor, *, transr: str = "T", uplo: str = "U",
             math: str = "fp32") -> torch.Tensor:
    """New RFP tensor holding the Cholesky factor of C (same layout as
    curfp_b200.spftrf leaves it); raises LinAlgError if C is not positive
    definite."""
    return _Cholesky.apply(C, transr, uplo, math)


def solve(L: torch.Tensor, B: torch.Tensor, *, transr: str = "T",
          uplo: str = "U") -> torch.Tensor:
    """X = (L L^T)^-1 B for the RFP factor L, B of shape (n,) or (n, nrhs)."""
    return _Solve.apply(L, B, transr, uplo)


def log_diag_sum(L: torch.Tensor, *, transr: str = "T", uplo: str = "U") -> torch.Tensor:
    """sum_i log L_ii of an RFP factor (half the log-determinant of L L^T)."""
    n = _check_rfp(L, "L")
    idx = _diag_idx(n, transr, uplo, L.device)
    return torch.log(L.index_select(0, idx)).sum()


def nll(X: torch.Tensor, s, sigma2, y: torch.Tensor, *, transr: str = "T",
        uplo: str = "U", math: str = "fp32", fused: bool = True,
        refine: int = 3) -> torch.Tensor:
    """1/2 y^T C^-1 y + sum log diag(L), C = s X X^T + sigma2 I = L L^T.
    ``refine``: at most this many FP64-residual corrections of alpha = C^-1 y
    (fused form)."""
    if fused:
        return _GpNll.apply(X, s, sigma2, y, transr, uplo, math, refine)
    C = ssfrk(X, s, transr=transr, uplo=uplo, math=math)
    C = add_to_diagonal(C, sigma2, transr=transr, uplo=uplo)
    L = cholesky(C, transr=transr, uplo=uplo, math=math)
    alpha = solve(L, y, transr=transr, uplo=uplo)
    return 0.5 * torch.dot(y, alpha) + log_diag_sum(L, transr=transr, uplo=uplo)
