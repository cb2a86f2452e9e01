#!/usr/bin/env python
"""Scale workloads of the RFP path on one GPU (helpers of tests/test_scale_gpu.py).

C2   plain FP32 drop-in at n in {32767, 32768}, k = 1024, all 8 variants:
     ssfrk, spftrf, spftrs (64 RHS) and spftri through the C ABI, beside the
     reference's own GPU build (oracle/_ref/libcurfp_ref.so, cuBLAS/cuSOLVER)
     on the same input, with FP64 checks of both: ||C - L L^T||_F / ||C||_F,
     solve backward error, inverse residual, ours-vs-reference differences.
C3   precision form at n = 65536, k = 2048, 256 RHS, per shift lambda:
     split-BF16 ssfrk + spftrf + FP64-residual refined spftrs against the
     FP32 (SIMT) form and the drop-in, errors against the exact FP64 solution.
C5   n = 131072, k = 4096, lambda = 1e-2: split-BF16 ssfrk + spftrf + refined
     spftrs (64 RHS), then the fused GP NLL forward + backward (X = A, s = 1,
     sigma2 = lambda), with the loss and gradient against exact FP64 values.
next the routines beyond the Cholesky path at n = 32768 (slansf, spfcon,
     ssfmv, ssfmm with 64 RHS, ssfr, ssfr2) and the FP64 twins at n = 16384
     (dsfrk k = 512, dpftrf, dpftrs with 64 RHS, dpftri), beside the
     reference build.

Each run_* function returns one result dict per case (timings, errors); the
tests assert the stated bounds on it and, when CURFP_SCALE_LOG names a file,
append it there as a JSON line (the numbers summarised under profiles/).

The FP64 oracle of C3 / C5 is exact and needs no n x n factorization: for
C = A A^T + lam I with A (n x k, its FP32 values, n > k) the Woodbury
identity gives C^-1 B = (B - A G^-1 A^T B) / lam with G = A^T A + lam I
(k x k, FP64 Cholesky), the residual B - C X = B - A (A^T X) - lam X, and
from the eigenvalues s_i of A^T A: ||C||_2 = max s_i + lam,
cond_2(C) = ||C||_2 / lam, log det C = (n-k) log lam + sum log(s_i + lam),
tr C^-1 = (n-k)/lam + sum 1/(s_i + lam).  Inputs are seeded numpy
default_rng draws: A ~ N(0,1)/sqrt(k) (n x k float32), B ~ N(0,1).
Timing: CUDA events on the default stream (the library handle's stream),
`warmup` untimed runs then the median of `reps`; the input of each in-place
routine is restored (untimed) before every run.
"""
from __future__ import annotations

import ctypes
import os
import json
import math
import statistics
import sys
import time
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import curfp_b200 as curfp  # noqa: E402
from curfp_b200 import autograd as ag  # noqa: E402
from curfp_b200 import precision  # noqa: E402

VARIANTS = [(tr, ul) for tr in (0, 1) for ul in (0, 1)]  # transr 0=N 1=T, uplo 0=L 1=U
NAME = lambda tr, ul: "NT"[tr] + "LU"[ul]  # noqa: E731


def vp(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def chol_flops(n: int) -> float:
    return n ** 3 / 3.0 + n ** 2 / 2.0 + n / 6.0


def emit(d: dict) -> None:
    """Append a result to the file named by CURFP_SCALE_LOG (if set)."""
    out = os.environ.get("CURFP_SCALE_LOG")
    if out:
        with open(out, "a") as f:
            f.write(json.dumps(d) + "\n")


class Ours:
    """This library through its C ABI (the drop-in boundary).  math=None runs
    the drop-in entry points in the handle's math mode; 0 / 1 select the
    arithmetic per call through the *Ex entry points."""

    def __init__(self):
        self.h = curfp._get_handle()
        self.lib = self.h._lib

    def ssfrk(self, tr, ul, n, k, A, C, math=None):
        a, b = ctypes.c_float(1.0), ctypes.c_float(0.0)
        if math is None:
            st = self.lib.curfpSsfrk(self.h.ptr, tr, ul, 1, n, k, ctypes.byref(a), vp(A), k,
                                     ctypes.byref(b), vp(C))
        else:
            st = self.lib.curfpSsfrkEx(self.h.ptr, tr, ul, 1, n, k, ctypes.byref(a), vp(A), k,
                                       ctypes.byref(b), vp(C), math)
        assert st == 0, st

    def add_diag(self, tr, ul, n, v, C):
        assert self.lib.curfpSaddToDiagonal(self.h.ptr, tr, ul, n, ctypes.c_float(v), vp(C)) == 0

    def spftrf(self, tr, ul, n, C, math=None):
        info = ctypes.c_int(0)
        if math is None:
            st = self.lib.curfpSpftrf(self.h.ptr, tr, ul, n, vp(C), ctypes.byref(info))
        else:
            st = self.lib.curfpSpftrfEx(self.h.ptr, tr, ul, n, vp(C), ctypes.byref(info), math)
        assert st == 0 and info.value == 0, (st, info.value)

    def spftrs(self, tr, ul, n, nrhs, F, X):
        assert self.lib.curfpSpftrs(self.h.ptr, tr, ul, n, nrhs, vp(F), vp(X), n) == 0

    def refine(self, tr, ul, n, nrhs, C, F, X, max_iter):
        it = ctypes.c_int(0)
        st = self.lib.curfpSpftrsRefine(self.h.ptr, tr, ul, n, nrhs, vp(C), vp(F), vp(X), n,
                                        max_iter, ctypes.byref(it))
        assert st == 0, st
        return it.value

    def spftri(self, tr, ul, n, F):
        assert self.lib.curfpSpftri(self.h.ptr, tr, ul, n, vp(F)) == 0

    def stfttr(self, tr, ul, n, arf, D):
        assert self.lib.curfpSstfttr(self.h.ptr, tr, ul, n, vp(arf), vp(D), n) == 0

    def slansf(self, norm, tr, ul, n, C):
        out = ctypes.c_float(0.0)
        assert self.lib.curfpSlansf(self.h.ptr, norm, tr, ul, n, vp(C), ctypes.byref(out)) == 0
        return float(out.value)

    def spfcon(self, tr, ul, n, F, anorm):
        out = ctypes.c_float(0.0)
        assert self.lib.curfpSpfcon(self.h.ptr, tr, ul, n, vp(F), ctypes.c_float(anorm),
                                    ctypes.byref(out)) == 0
        return float(out.value)

    def release(self):
        assert self.lib.curfpReleaseWorkspace(self.h.ptr) == 0

    def mode(self, m: str):
        """Context manager: the handle's math mode set to m ("bf16x3" /
        "fp32") inside the block."""
        ours = self

        class _M:
            def __enter__(self_):
                self_.prev = ours.h.get_math_mode()
                ours.h.set_math_mode(m)

            def __exit__(self_, *exc):
                ours.h.set_math_mode(self_.prev)
                return False
        return _M()


def cuda_ms(fn, prep=None, warmup=2, reps=5):
    """Median device milliseconds of fn() over reps runs after warmup runs."""
    ts = []
    for i in range(warmup + reps):
        if prep is not None:
            prep()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        if i >= warmup:
            ts.append(e0.elapsed_time(e1))
    return statistics.median(ts)


def rate(ms, flops=None, nbytes=None):
    d = {"ms": round(ms, 3)}
    if flops is not None:
        d["tflops"] = round(flops / (ms * 1e-3) / 1e12, 3)
    if nbytes is not None:
        d["gbs"] = round(nbytes / (ms * 1e-3) / 1e9, 1)
    return d


def gen_A(n, k, seed):
    rng = np.random.default_rng(seed)
    A = (rng.standard_normal((n, k), dtype=np.float32) / np.float32(math.sqrt(k)))
    return torch.from_numpy(A).cuda()


def gen_B(n, nrhs, seed):
    """(nrhs, n) row-major = the column-major n x nrhs block of the C ABI."""
    rng = np.random.default_rng(seed)
    return torch.from_numpy(rng.standard_normal((nrhs, n), dtype=np.float32)).cuda()


# ---------------------------------------------------------------------------
# FP64 checks
# ---------------------------------------------------------------------------

class GramOracle:
    """Exact FP64 facts of C = A A^T + lam I (A n x k, n > k) from A's Gram
    matrix (Woodbury identity)."""

    def __init__(self, A32, lam):
        n, k = A32.shape
        assert n > k
        self.n, self.k, self.lam = n, k, float(lam)
        self.A = A32.double()
        G = self.A.T @ self.A
        self.s = torch.linalg.eigvalsh(G)
        G.diagonal().add_(self.lam)
        self.Lg = torch.linalg.cholesky(G)
        del G
        self.norm2 = float(self.s.max()) + self.lam
        self.cond2 = self.norm2 / self.lam

    def apply(self, X):  # C X
        return self.A @ (self.A.T @ X) + self.lam * X

    def solve(self, B):  # C^-1 B
        u = torch.cholesky_solve(self.A.T @ B, self.Lg)
        return (B - self.A @ u) / self.lam

    def logdet(self) -> float:
        return (self.n - self.k) * math.log(self.lam) + float(torch.log(self.s + self.lam).sum())

    def trace_inv(self) -> float:
        return (self.n - self.k) / self.lam + float((1.0 / (self.s + self.lam)).sum())

    def trace_ata_cinv(self) -> float:  # tr(A^T C^-1 A)
        return float((self.s / (self.s + self.lam)).sum())

    def cinv_a(self):  # C^-1 A = A G^-1
        return torch.cholesky_solve(self.A.T.contiguous(), self.Lg).T


def solve_errors(orc: GramOracle, B32, X32) -> dict:
    """Normwise backward error max_j ||b_j - C x_j|| / (||C||_2 ||x_j|| + ||b_j||)
    and forward error max_j ||x_j - x*_j|| / ||x*_j|| against the exact C."""
    B = B32.double().T
    X = X32.double().T
    R = B - orc.apply(X)
    berr = (R.norm(dim=0) / (orc.norm2 * X.norm(dim=0) + B.norm(dim=0))).max()
    X64 = orc.solve(B)
    ferr = ((X - X64).norm(dim=0) / X64.norm(dim=0)).max()
    return {"backward": float(berr), "forward": float(ferr)}


def dense_sym(ours: Ours, tr, ul, n, arf):
    """FP64 n x n symmetric matrix of an RFP array (exact widening)."""
    D = torch.zeros(n, n, device="cuda")
    ours.stfttr(tr, ul, n, arf, D)
    S = D.double()
    del D
    S += S.T.clone()
    S.diagonal().mul_(0.5)
    return S


def dense_tri(ours: Ours, tr, ul, n, arf):
    """FP64 stored triangle of an RFP factor: L (uplo=L, row-major lower) or
    U (uplo=U, row-major upper)."""
    D = torch.zeros(n, n, device="cuda")
    ours.stfttr(tr, ul, n, arf, D)
    T = D.double()
    del D
    return T


def factor_berr(S, T, ul) -> float:
    P = (T.T @ T) if ul == 1 else (T @ T.T)
    P -= S
    r = float(torch.linalg.norm(P) / torch.linalg.norm(S))
    del P
    return r


def solve_berr_dense(S, norm2, B32, X32) -> float:
    B = B32.double().T
    X = X32.double().T
    R = B - S @ X
    return float((R.norm(dim=0) / (norm2 * X.norm(dim=0) + B.norm(dim=0))).max())


def inverse_res(S, I_sym) -> float:
    """||C Z - I||_F / sqrt(n): RMS over columns of ||C z_j - e_j||."""
    P = S @ I_sym
    P.diagonal().sub_(1.0)
    r = float(torch.linalg.norm(P) / math.sqrt(S.shape[0]))
    del P
    return r


def rel_diff(a, b) -> float:
    return float(torch.linalg.norm((a - b).double()) / torch.linalg.norm(b.double()))


# ---------------------------------------------------------------------------
# C2: plain FP32 at scale, all variants, beside the reference build
# ---------------------------------------------------------------------------

def run_c2(n, tr, ul, mode="bf16x3", warmup=2, reps=5, with_ref=True) -> dict:
    """One C2 case: the drop-in routines in the handle math `mode` beside the
    reference build (when present) on the same input; timings are medians of
    `reps` runs after `warmup` (reps = 1, warmup = 0: one run each)."""
    from helpers import REF_LIB, RefLib
    ours = Ours()
    ref = RefLib() if (with_ref and REF_LIB.exists()) else None
    k, nrhs, shift = 1024, 64, 1.0
    A = gen_A(n, k, seed=n)
    B0 = gen_B(n, nrhs, seed=n + 1)
    orc = GramOracle(A, shift)  # only for ||C||_2 of the exact matrix
    nt = n * (n + 1) // 2
    f = {"ssfrk": n * (n + 1) * float(k), "spftrf": chol_flops(n),
         "spftrs": 2.0 * n * n * nrhs, "spftri": 2.0 * n ** 3 / 3.0}
    by = {"ssfrk": 4.0 * n * k + 4.0 * nt, "spftrf": 8.0 * nt,
          "spftrs": 8.0 * nt + 16.0 * n * nrhs, "spftri": 8.0 * nt}
    res = {"config": "C2", "n": n, "k": k, "nrhs": nrhs, "shift": shift,
           "variant": NAME(tr, ul), "transr": "NT"[tr], "uplo": "LU"[ul], "math": mode,
           "timing": f"warmup {warmup}, median of {reps}",
           "ours": {}, "reference": {}, "errors": {}}
    C0 = torch.empty(nt, device="cuda")
    F = torch.empty_like(C0)
    X = torch.empty_like(B0)
    Z = torch.empty_like(C0)
    with ours.mode(mode):
        ms = cuda_ms(lambda: ours.ssfrk(tr, ul, n, k, A, C0), None, warmup, reps)
        res["ours"]["ssfrk"] = rate(ms, f["ssfrk"], by["ssfrk"])
        ours.add_diag(tr, ul, n, shift, C0)
        ms = cuda_ms(lambda: ours.spftrf(tr, ul, n, F), lambda: F.copy_(C0), warmup, reps)
        res["ours"]["spftrf"] = rate(ms, f["spftrf"], by["spftrf"])
        ms = cuda_ms(lambda: ours.spftrs(tr, ul, n, nrhs, F, X), lambda: X.copy_(B0),
                     warmup, reps)
        res["ours"]["spftrs"] = rate(ms, f["spftrs"], by["spftrs"])
        ms = cuda_ms(lambda: ours.spftri(tr, ul, n, Z), lambda: Z.copy_(F), warmup, reps)
        res["ours"]["spftri"] = rate(ms, f["spftri"], by["spftri"])
    t = res["ours"]
    t["chol_solve_tflops"] = round((f["spftrf"] + f["spftrs"]) /
                                   ((t["spftrf"]["ms"] + t["spftrs"]["ms"]) * 1e-3) / 1e12, 3)
    if ref is not None:
        Cr = torch.empty(nt, device="cuda")
        ms = cuda_ms(lambda: ref.ssfrk(tr, ul, 1, n, k, 1.0, A, k, 0.0, Cr), None, warmup, reps)
        res["reference"]["ssfrk"] = rate(ms, f["ssfrk"], by["ssfrk"])
        ours.add_diag(tr, ul, n, shift, Cr)
        res["errors"]["ssfrk_maxabs_ours_vs_ref"] = float((Cr - C0).abs().max())
        del Cr
        Fr = torch.empty_like(C0)
        Xr = torch.empty_like(B0)
        Zr = torch.empty_like(C0)
        infos = []

        def rf():
            st, info = ref.spftrf(tr, ul, n, Fr)
            assert st == 0, st
            infos.append(info)
        ms = cuda_ms(rf, lambda: Fr.copy_(C0), warmup, reps)
        res["reference"]["spftrf"] = rate(ms, f["spftrf"], by["spftrf"])
        res["reference_info"] = infos[-1]
        ms = cuda_ms(lambda: ref.spftrs(tr, ul, n, nrhs, Fr, Xr, n), lambda: Xr.copy_(B0),
                     warmup, reps)
        res["reference"]["spftrs"] = rate(ms, f["spftrs"], by["spftrs"])
        ms = cuda_ms(lambda: ref.spftri(tr, ul, n, Zr), lambda: Zr.copy_(Fr), warmup, reps)
        res["reference"]["spftri"] = rate(ms, f["spftri"], by["spftri"])
        t = res["reference"]
        t["chol_solve_tflops"] = round(
            (f["spftrf"] + f["spftrs"]) /
            ((t["spftrf"]["ms"] + t["spftrs"]["ms"]) * 1e-3) / 1e12, 3)
        e = res["errors"]
        e["factor_rel_diff_ours_vs_ref"] = rel_diff(F, Fr)
        e["solve_rel_diff_ours_vs_ref"] = rel_diff(X, Xr)
        e["inverse_rel_diff_ours_vs_ref"] = rel_diff(Z, Zr)
    # FP64 checks on the stored FP32 matrix C0 (the input of both arms)
    S = dense_sym(ours, tr, ul, n, C0)
    e = res["errors"]
    arms = [("ours", F, X, Z)] + ([("reference", Fr, Xr, Zr)] if ref is not None else [])
    for name, Fa, Xa, Za in arms:
        T = dense_tri(ours, tr, ul, n, Fa)
        e[f"{name}_factor_backward"] = factor_berr(S, T, ul)
        del T
        e[f"{name}_solve_backward"] = solve_berr_dense(S, orc.norm2, B0, Xa)
        Zs = dense_sym(ours, tr, ul, n, Za)
        e[f"{name}_inverse_residual"] = inverse_res(S, Zs)
        del Zs
    del S, F, X, Z, C0, A, B0, orc
    if ref is not None:
        del Fr, Xr, Zr
    torch.cuda.empty_cache()
    return res


# ---------------------------------------------------------------------------
# C3: precision form vs plain at n = 65536
# ---------------------------------------------------------------------------

def breakdown(fn) -> dict:
    precision.profile_enable(True)
    fn()
    torch.cuda.synchronize()
    r = precision.profile_read()
    precision.profile_enable(False)
    return {k: round(v["ms"], 2) for k, v in r.items()}


def run_c3(lam, n=65536, k=2048, warmup=2, reps=5, max_iter=3) -> dict:
    """One C3 case (shift lam): the FP32 (SIMT) form, the drop-in in its
    default math mode, and the precision form (split-BF16 factor + FP64
    refined solve), each against the exact FP64 solution."""
    from types import SimpleNamespace
    args = SimpleNamespace(c3_n=n, c3_k=k, lam=[lam], warmup=warmup, reps=reps,
                           max_iter=max_iter)
    ours = Ours()
    n, k, nrhs = args.c3_n, args.c3_k, 256
    tr, ul = 1, 1
    nt = n * (n + 1) // 2
    A = gen_A(n, k, seed=65536)
    B0 = gen_B(n, nrhs, seed=65537)
    fl = chol_flops(n) + 2.0 * n * n * nrhs
    for lam in args.lam:
        orc = GramOracle(A, lam)
        res = {"config": "C3", "n": n, "k": k, "nrhs": nrhs, "lambda": lam, "variant": "TU",
               "cond2_exact": orc.cond2, "norm2_exact": orc.norm2,
               "timing": f"warmup {args.warmup}, median of {args.reps}",
               "metric": "Cholesky+solve TFLOP/s = (n^3/3 + n^2/2 + n/6 + 2 n^2 nrhs) / t"}
        for form, math_ in (("plain_fp32", 0), ("drop_in_default", None), ("split_bf16", 1)):
            C = torch.empty(nt, device="cuda")
            ms_s = cuda_ms(lambda: ours.ssfrk(tr, ul, n, k, A, C, math_), None,
                           args.warmup, args.reps)
            ours.add_diag(tr, ul, n, lam, C)
            F = torch.empty_like(C)
            X = torch.empty_like(B0)
            ms_f = cuda_ms(lambda: ours.spftrf(tr, ul, n, F, math_), lambda: F.copy_(C),
                           args.warmup, args.reps)
            iters = []
            if math_ != 1:
                with ours.mode("fp32" if math_ == 0 else "bf16x3"):
                    ms_x = cuda_ms(lambda: ours.spftrs(tr, ul, n, nrhs, F, X),
                                   lambda: X.copy_(B0), args.warmup, args.reps)
            else:
                ms_x = cuda_ms(lambda: iters.append(
                    ours.refine(tr, ul, n, nrhs, C, F, X, args.max_iter)),
                    lambda: X.copy_(B0), args.warmup, args.reps)
            d = {"ssfrk": rate(ms_s, n * (n + 1) * float(k)),
                 "spftrf": rate(ms_f, chol_flops(n)),
                 "spftrs" if math_ != 1 else "spftrs_refined": rate(ms_x, 2.0 * n * n * nrhs),
                 "chol_solve": rate(ms_f + ms_x, fl)}
            if iters:
                d["refine_corrections"] = iters[-1]
            d["errors_vs_fp64"] = solve_errors(orc, B0, X)
            d.update(conditioning(ours, tr, ul, n, C, F))
            # the stored matrix against the exact one on 512 sampled rows
            d["ssfrk_rel_err_sampled"] = ssfrk_sample_err(ours, tr, ul, n, C, orc, 512)
            d["breakdown_ms"] = breakdown(lambda: (F.copy_(C), ours.spftrf(tr, ul, n, F, math_)))
            res[form] = d
            del C, F, X
            torch.cuda.empty_cache()
            ours.release()
        res["precision_over_plain"] = round(res["split_bf16"]["chol_solve"]["tflops"] /
                                            res["plain_fp32"]["chol_solve"]["tflops"], 3)
        del orc
        torch.cuda.empty_cache()
    return res


def conditioning(ours: Ours, tr, ul, n, C, F) -> dict:
    """1-norm condition estimate of the stored matrix: slansf('1') of C and
    spfcon on its factor F (both timed once, host result)."""
    t0 = time.perf_counter()
    anorm = ours.slansf(1, tr, ul, n, C)
    t1 = time.perf_counter()
    rc = ours.spfcon(tr, ul, n, F, anorm)
    t2 = time.perf_counter()
    return {"anorm_1": anorm, "rcond_spfcon": rc, "cond1_est": (1.0 / rc) if rc else None,
            "slansf_ms": round((t1 - t0) * 1e3, 2), "spfcon_ms": round((t2 - t1) * 1e3, 2)}


def ssfrk_sample_err(ours: Ours, tr, ul, n, C, orc: GramOracle, nrows: int) -> float:
    """max |C_stored - C_exact| / max |C_exact| over nrows sampled rows."""
    rows = torch.from_numpy(np.sort(np.random.default_rng(5).choice(n, nrows, replace=False)))
    rows = rows.cuda()
    Ce = orc.A[rows] @ orc.A.T  # nrows x n
    Ce[torch.arange(nrows, device="cuda"), rows] += orc.lam
    got = torch.empty_like(Ce)
    # row r of the symmetric matrix from the RFP array: element (r, j) lives
    # at the RFP offset of logical lower element (max, min)
    offs = rfp_offsets(tr, ul, n, rows)
    got.copy_(C[offs].double())
    err = float((got - Ce).abs().max() / Ce.abs().max())
    return err


def rfp_offsets(tr, ul, n, rows):
    """RFP offsets (int64, nrows x n) of the symmetric matrix's rows `rows`:
    the lower element (max(r, j), min(r, j)) of the logical factor, through the
    block geometry of the variant (rfp_diag_indices gives the diagonal, the
    blocks' strides follow from it)."""
    lower = ul == 0
    if n % 2:
        n1, n2 = ((n + 1) // 2, n // 2) if lower else (n // 2, (n + 1) // 2)
    else:
        n1 = n2 = n // 2
    kk = n // 2
    N = n
    if n % 2:
        if tr == 0:
            g = ((0, 1, N), (n1, 1, N), (N, N, 1)) if lower else ((n2, 1, N), (0, N, 1), (n1, N, 1))
        else:
            g = (((0, n1, 1), (n1 * n1, n1, 1), (1, 1, n1)) if lower else
                 ((n2 * n2, n2, 1), (0, 1, n2), (n1 * n2, 1, n2)))
    else:
        if tr == 0:
            g = (((1, 1, N + 1), (kk + 1, 1, N + 1), (0, N + 1, 1)) if lower else
                 ((kk + 1, 1, N + 1), (0, N + 1, 1), (kk, N + 1, 1)))
        else:
            g = (((kk, kk, 1), (kk * (kk + 1), kk, 1), (0, 1, kk)) if lower else
                 ((kk * (kk + 1), kk, 1), (0, 1, kk), (kk * kk, 1, kk)))
    r = rows.view(-1, 1).long()
    j = torch.arange(n, device=rows.device).view(1, -1)
    p = torch.maximum(r, j)
    q = torch.minimum(r, j)
    o11 = g[0][0] + p * g[0][1] + q * g[0][2]
    o21 = g[1][0] + (p - n1) * g[1][1] + q * g[1][2]
    o22 = g[2][0] + (p - n1) * g[2][1] + (q - n1) * g[2][2]
    return torch.where(q < n1, torch.where(p < n1, o11, o21), o22)


# ---------------------------------------------------------------------------
# C5: n = 131072 precision pipeline + fused NLL fwd/bwd
# ---------------------------------------------------------------------------

def run_c5(n=131072, k=4096, warmup=1, reps=3, max_iter=3, nll=True, nll_warmup=1,
           nll_reps=3) -> dict:
    """The C5 pipeline (split-BF16 ssfrk + spftrf + refined spftrs) and,
    with nll, the fused GP NLL forward + backward, against exact FP64."""
    from types import SimpleNamespace
    args = SimpleNamespace(c5_n=n, c5_k=k, warmup=warmup, reps=reps, max_iter=max_iter,
                           nll_warmup=nll_warmup, nll_reps=nll_reps)
    ours = Ours()
    n, k, nrhs, lam = args.c5_n, args.c5_k, 64, 1e-2
    tr, ul = 1, 1
    nt = n * (n + 1) // 2
    A = gen_A(n, k, seed=131072)
    B0 = gen_B(n, nrhs, seed=131073)
    orc = GramOracle(A, lam)
    res = {"config": "C5", "n": n, "k": k, "nrhs": nrhs, "lambda": lam, "variant": "TU",
           "cond2_exact": orc.cond2, "rfp_gb_per_copy": round(4.0 * nt / 1e9, 2),
           "timing": f"warmup {args.warmup}, median of {args.reps}"}
    C = torch.empty(nt, device="cuda")
    ms_s = cuda_ms(lambda: ours.ssfrk(tr, ul, n, k, A, C, 1), None, args.warmup, args.reps)
    ours.add_diag(tr, ul, n, lam, C)
    F = torch.empty_like(C)
    X = torch.empty_like(B0)
    ms_f = cuda_ms(lambda: ours.spftrf(tr, ul, n, F, 1), lambda: F.copy_(C), args.warmup,
                   args.reps)
    iters = []
    ms_x = cuda_ms(lambda: iters.append(ours.refine(tr, ul, n, nrhs, C, F, X, args.max_iter)),
                   lambda: X.copy_(B0), args.warmup, args.reps)
    fl = chol_flops(n) + 2.0 * n * n * nrhs
    res["split_bf16"] = {
        "ssfrk": rate(ms_s, n * (n + 1) * float(k)),
        "spftrf": rate(ms_f, chol_flops(n)),
        "spftrs_refined": rate(ms_x, 2.0 * n * n * nrhs),
        "chol_solve": rate(ms_f + ms_x, fl),
        "pipeline_ms": round(ms_s + ms_f + ms_x, 1),
        "refine_corrections": iters[-1],
        "errors_vs_fp64": solve_errors(orc, B0, X),
        **conditioning(ours, tr, ul, n, C, F),
        "ssfrk_rel_err_sampled": ssfrk_sample_err(ours, tr, ul, n, C, orc, 256),
        "breakdown_ms": breakdown(lambda: (F.copy_(C), ours.spftrf(tr, ul, n, F, 1))),
        "peak_mem_gb": round(torch.cuda.max_memory_allocated() / 1e9, 1)}
    del C, F, X
    torch.cuda.empty_cache()
    ours.release()
    if nll:
        res["nll"] = nll_c5(orc, A, lam, args)
    del A, B0, orc
    torch.cuda.empty_cache()
    ours.release()
    return res


def nll_c5(orc: GramOracle, A, lam, args) -> dict:
    """Fused GP NLL (X = A, s = 1, sigma2 = lam) forward + backward, against
    the exact FP64 loss and gradient."""
    n, k = A.shape
    y = torch.from_numpy(np.random.default_rng(7).standard_normal(n, dtype=np.float32)).cuda()
    out = {"workload": f"loss = 1/2 y^T C^-1 y + sum log diag L, C = s X X^T + sigma2 I, "
                       f"X = A ({n} x {k}), s = 1, sigma2 = {lam}; fused form, split-BF16"}
    holder = {}

    def step():
        Xt = A.clone().requires_grad_(True)
        st = torch.tensor(1.0, device="cuda", requires_grad=True)
        vt = torch.tensor(lam, device="cuda", requires_grad=True)
        loss = ag.nll(Xt, st, vt, y, math="bf16x3", fused=True)
        loss.backward()
        holder.update(loss=loss.detach(), gx=Xt.grad, gs=st.grad, gv=vt.grad)

    out["fwd_bwd_ms"] = round(cuda_ms(step, lambda: holder.clear(), args.nll_warmup,
                                      args.nll_reps), 1)
    loss64, gx64, gs64, gv64 = nll_exact(orc, y)
    out["errors_vs_fp64"] = {
        "loss": abs(float(holder["loss"]) - loss64) / abs(loss64),
        "grad_X": float(torch.linalg.norm(holder["gx"].double() - gx64) /
                        torch.linalg.norm(gx64)),
        "grad_s": abs(float(holder["gs"]) - gs64) / abs(gs64),
        "grad_sigma2": abs(float(holder["gv"]) - gv64) / abs(gv64)}
    out["peak_mem_gb"] = round(torch.cuda.max_memory_allocated() / 1e9, 1)
    return out


# ---------------------------------------------------------------------------
# The routines beyond the Cholesky path: norms, condition estimate,
# symmetric multiplies, rank updates, and the FP64 twins
# ---------------------------------------------------------------------------

def run_next(n=32768, nd=16384, warmup=2, reps=5) -> dict:
    """The routines beyond the Cholesky path beside the reference build."""
    from types import SimpleNamespace

    from helpers import REF_LIB, RefLib
    args = SimpleNamespace(next_n=n, next_nd=nd, warmup=warmup, reps=reps)
    ours = Ours()
    ref = RefLib() if REF_LIB.exists() else None
    lib, h = ours.lib, ours.h.ptr
    n, k, tr, ul = args.next_n, 1024, 1, 1
    nt = n * (n + 1) // 2
    A = gen_A(n, k, seed=n + 3)
    C = torch.empty(nt, device="cuda")
    ours.ssfrk(tr, ul, n, k, A, C)
    ours.add_diag(tr, ul, n, 1.0, C)
    F = C.clone()
    ours.spftrf(tr, ul, n, F)
    W, R = args.warmup, args.reps
    res = {"config": "next-ops", "n": n, "variant": "TU",
           "timing": f"warmup {W}, median of {R}", "ops": {}}
    o = res["ops"]
    fl = ctypes.c_float(0.0)

    def both(name, ours_fn, ref_fn, flops=None, nbytes=None, prep=None):
        d = {"ours": rate(cuda_ms(ours_fn, prep, W, R), flops, nbytes)}
        if ref is not None and ref_fn is not None:
            d["reference"] = rate(cuda_ms(ref_fn, prep, W, R), flops, nbytes)
        o[name] = d

    for norm, nm in ((0, "slansf_max"), (1, "slansf_one"), (2, "slansf_fro")):
        both(nm, lambda: lib.curfpSlansf(h, norm, tr, ul, n, vp(C), ctypes.byref(fl)),
             (lambda: ref.slansf(norm, tr, ul, n, C)) if ref else None, nbytes=4.0 * nt)
        o[nm]["value_ours"] = ours.slansf(norm, tr, ul, n, C)
        if ref:
            o[nm]["value_reference"] = ref.slansf(norm, tr, ul, n, C)[1]
    anorm = ours.slansf(1, tr, ul, n, C)
    both("spfcon", lambda: ours.spfcon(tr, ul, n, F, anorm),
         (lambda: ref.spfcon(tr, ul, n, F, anorm)) if ref else None)
    o["spfcon"]["rcond_ours"] = ours.spfcon(tr, ul, n, F, anorm)
    if ref:
        o["spfcon"]["rcond_reference"] = ref.spfcon(tr, ul, n, F, anorm)[1]
    x = torch.randn(n, device="cuda")
    y = torch.zeros(n, device="cuda")
    a1, b0 = ctypes.c_float(1.0), ctypes.c_float(0.0)
    both("ssfmv", lambda: lib.curfpSsfmv(h, tr, ul, n, ctypes.byref(a1), vp(C), vp(x), 1,
                                        ctypes.byref(b0), vp(y), 1),
         (lambda: ref.ssfmv(tr, ul, n, 1.0, C, x, 1, 0.0, y, 1)) if ref else None,
         flops=2.0 * n * n, nbytes=4.0 * nt)
    Bm = torch.randn(64, n, device="cuda")
    Ym = torch.zeros(64, n, device="cuda")
    both("ssfmm_64", lambda: lib.curfpSsfmm(h, tr, ul, 0, n, 64, ctypes.byref(a1), vp(C),
                                           vp(Bm), n, ctypes.byref(b0), vp(Ym), n),
         (lambda: ref.ssfmm(tr, ul, 0, n, 64, 1.0, C, Bm, n, 0.0, Ym, n)) if ref else None,
         flops=2.0 * n * n * 64)
    Cw = C.clone()
    both("ssfr", lambda: lib.curfpSsfr(h, tr, ul, n, ctypes.byref(a1), vp(x), 1, vp(Cw)),
         (lambda: ref.ssfr(tr, ul, n, 1.0, x, 1, Cw)) if ref else None, nbytes=8.0 * nt)
    both("ssfr2", lambda: lib.curfpSsfr2(h, tr, ul, n, ctypes.byref(a1), vp(x), 1, vp(y), 1,
                                        vp(Cw)),
         (lambda: ref.ssfr2(tr, ul, n, 1.0, x, 1, y, 1, Cw)) if ref else None, nbytes=8.0 * nt)
    del Cw, C, F, A
    torch.cuda.empty_cache()
    # FP64 twins
    nd, kd = args.next_nd, 512
    ntd = nd * (nd + 1) // 2
    Ad = gen_A(nd, kd, seed=nd).double()
    Cd = torch.empty(ntd, device="cuda", dtype=torch.float64)
    ad, bd = ctypes.c_double(1.0), ctypes.c_double(0.0)
    info = ctypes.c_int(0)
    both("dsfrk", lambda: lib.curfpDsfrk(h, tr, ul, 1, nd, kd, ctypes.byref(ad), vp(Ad), kd,
                                        ctypes.byref(bd), vp(Cd)),
         (lambda: ref.dsfrk(tr, ul, 1, nd, kd, 1.0, Ad, kd, 0.0, Cd)) if ref else None,
         flops=nd * (nd + 1) * float(kd))
    import curfp_b200 as cf
    cf.add_to_diagonal(Cd, 1.0)
    Fd = torch.empty_like(Cd)
    both("dpftrf", lambda: lib.curfpDpftrf(h, tr, ul, nd, vp(Fd), ctypes.byref(info)),
         (lambda: ref.dpftrf(tr, ul, nd, Fd)) if ref else None, flops=chol_flops(nd),
         prep=lambda: Fd.copy_(Cd))
    Fd.copy_(Cd)
    lib.curfpDpftrf(h, tr, ul, nd, vp(Fd), ctypes.byref(info))
    Bd = torch.randn(64, nd, device="cuda", dtype=torch.float64)
    Xd = torch.empty_like(Bd)
    both("dpftrs_64", lambda: lib.curfpDpftrs(h, tr, ul, nd, 64, vp(Fd), vp(Xd), nd),
         (lambda: ref.dpftrs(tr, ul, nd, 64, Fd, Xd, nd)) if ref else None,
         flops=2.0 * nd * nd * 64, prep=lambda: Xd.copy_(Bd))
    Zd = torch.empty_like(Fd)
    both("dpftri", lambda: lib.curfpDpftri(h, tr, ul, nd, vp(Zd)),
         (lambda: ref.dpftri(tr, ul, nd, Zd)) if ref else None, flops=2.0 * nd ** 3 / 3.0,
         prep=lambda: Zd.copy_(Fd))
    res["fp64_n"] = nd
    del Ad, Cd, Fd, Bd, Xd, Zd, x, y, Bm, Ym
    torch.cuda.empty_cache()
    return res


def nll_exact(orc: GramOracle, y):
    """Exact FP64 loss and gradients (X, s, sigma2) of the GP NLL at X = A,
    s = 1, sigma2 = lam:  alpha = C^-1 y, loss = 1/2 y^T alpha + 1/2 log det C,
    dX = C^-1 A - alpha (A^T alpha)^T, ds = 1/2 (tr(A^T C^-1 A) - |A^T alpha|^2),
    dsigma2 = 1/2 (tr C^-1 - |alpha|^2)."""
    y64 = y.double()
    alpha = orc.solve(y64[:, None])[:, 0]
    loss64 = 0.5 * float(y64 @ alpha) + 0.5 * orc.logdet()
    ata = orc.A.T @ alpha
    gx64 = orc.cinv_a() - alpha[:, None] * ata[None, :]
    gs64 = 0.5 * (orc.trace_ata_cinv() - float(ata @ ata))
    gv64 = 0.5 * (orc.trace_inv() - float(alpha @ alpha))
    return loss64, gx64, gs64, gv64
