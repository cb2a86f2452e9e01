"""Parity at the scale workloads, on the GPU (helpers in tests/scale_lib.py).

C2: n in {32767, 32768}, k = 1024, A ~ N(0,1)/sqrt(k), shift 1.0, all 8
variants: ssfrk, spftrf, spftrs (64 RHS) and spftri through the C ABI beside
the reference's own GPU build (oracle/_ref) on the same device inputs, in the
handle's default math mode (split-BF16 tensor-core contractions) and, for two
variants, in the FP32 SIMT mode.  Stated bounds: identical info (0); our
factor / solve / inverse agree with the reference's to 1e-4 relative
(Frobenius); our FP64 backward errors ||C - L L^T||_F / ||C||_F, solve
max_j ||b_j - C x_j|| / (||C||_2 ||x_j|| + ||b_j||) and inverse residual
||C Z - I||_F / sqrt(n) are within 2x of the reference's (absolute bounds
5e-6 / 1e-6 / 5e-5 when the reference build is absent).  Reference pins these
extend: python_tests/test_vs_lapack.py:133-152, python_tests/test_spftrs.py:73-87
(n <= 512 there).

C3: n = 65536, k = 2048, 256 RHS, lambda in {1e-1, 1e-3}: the precision form's
solve backward error against the exact FP64 matrix (Woodbury) is <= the
FP32 (SIMT) form's and <= the drop-in's.

C5: n = 131072, k = 4096, lambda = 1e-2 (34.4 GB per RFP copy): split-BF16
ssfrk + spftrf + refined spftrs, backward error <= 1e-6 against the exact
matrix; the fused GP NLL forward + backward: loss within 1e-5, gradients to
s and sigma2 within 1e-4 and to X within 2e-3 of the exact FP64 values (the
d = 4096 FP32 solves for C^-1 X carry cond * u = 2.6e-4 at cond 4.4e3; the
1e-4 gradient target holds at the n = 8192 workload, test_autograd_gpu.py).

With CURFP_SCALE_LOG=<file> every case is timed (median of 5 after 2
warm-up runs) and its result appended to <file> as a JSON line."""
import os

import pytest
import torch

import scale_lib as S
from helpers import REF_LIB

TIMED = bool(os.environ.get("CURFP_SCALE_LOG"))
W, R = (2, 5) if TIMED else (0, 1)

C2_CASES = ([(n, tr, ul, "bf16x3") for n in (32768, 32767) for tr in (0, 1) for ul in (0, 1)] +
            [(32768, 1, 1, "fp32"), (32768, 0, 0, "fp32")])


@pytest.mark.gpu
@pytest.mark.parametrize("n,tr,ul,mode", C2_CASES,
                         ids=[f"{n}-{'NT'[t]}{'LU'[u]}-{m}" for n, t, u, m in C2_CASES])
def test_c2_vs_reference_build(curfp, n, tr, ul, mode):
    res = S.run_c2(n, tr, ul, mode=mode, warmup=W, reps=R)
    S.emit(res)
    e = res["errors"]
    if REF_LIB.exists():
        assert res["reference_info"] == 0
        for key in ("factor_rel_diff_ours_vs_ref", "solve_rel_diff_ours_vs_ref",
                    "inverse_rel_diff_ours_vs_ref"):
            assert e[key] <= 1e-4, (key, e[key])
        assert e["ours_factor_backward"] <= 2 * e["reference_factor_backward"] + 1e-7, e
        assert e["ours_solve_backward"] <= 2 * e["reference_solve_backward"] + 1e-8, e
        assert e["ours_inverse_residual"] <= 2 * e["reference_inverse_residual"] + 1e-6, e
    else:
        assert e["ours_factor_backward"] <= 5e-6, e
        assert e["ours_solve_backward"] <= 1e-6, e
        assert e["ours_inverse_residual"] <= 5e-5, e


@pytest.mark.gpu
@pytest.mark.parametrize("lam", [1e-1, 1e-3])
def test_c3_precision_form(curfp, lam):
    res = S.run_c3(lam, warmup=W, reps=R)
    S.emit(res)
    prec = res["split_bf16"]["errors_vs_fp64"]["backward"]
    assert prec <= res["plain_fp32"]["errors_vs_fp64"]["backward"], res
    assert prec <= res["drop_in_default"]["errors_vs_fp64"]["backward"], res
    assert res["split_bf16"]["refine_corrections"] >= 1


@pytest.mark.gpu
def test_c5_large_n(curfp):
    res = S.run_c5(warmup=min(W, 1), reps=min(R, 3), nll_warmup=min(W, 1), nll_reps=min(R, 3))
    S.emit(res)
    assert res["split_bf16"]["errors_vs_fp64"]["backward"] <= 1e-6, res
    e = res["nll"]["errors_vs_fp64"]
    assert e["loss"] <= 1e-5, e
    assert e["grad_s"] <= 1e-4 and e["grad_sigma2"] <= 1e-4, e
    assert e["grad_X"] <= 2e-3, e


@pytest.mark.gpu
def test_next_ops_vs_reference_build(curfp):
    res = S.run_next(warmup=W, reps=R)
    S.emit(res)
    o = res["ops"]
    if REF_LIB.exists():
        for nm in ("slansf_max", "slansf_one", "slansf_fro"):
            a, b = o[nm]["value_ours"], o[nm]["value_reference"]
            assert abs(a - b) <= 1e-5 * abs(b), (nm, a, b)
        a, b = o["spfcon"]["rcond_ours"], o["spfcon"]["rcond_reference"]
        assert abs(a - b) <= 1e-3 * abs(b), (a, b)
    torch.cuda.empty_cache()


@pytest.mark.gpu
def test_c5_cholesky_adjoint_in_rfp(curfp):
    """curfpSpftrfBackward at n = 131072 (34.4 GB per RFP array): the factor
    and the cotangent (updated in place) are the only n-squared arrays.  With
    Lbar = L (f = 1/2 tr A) the result is 1/2 on the diagonal and 0
    elsewhere: max |Abar - 1/2 I| <= 1e-4."""
    import ctypes
    n, k, lam = 131072, 4096, 1e-2
    A = S.gen_A(n, k, seed=131072)
    L = torch.empty(n * (n + 1) // 2, device="cuda")
    curfp.ssfrk(A, L)
    del A
    curfp.add_to_diagonal(L, lam)
    assert curfp.spftrf(L) == 0
    G = L.clone()
    h = curfp._get_handle()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    st = h._lib.curfpSpftrfBackward(h.ptr, 1, 1, n, ctypes.c_void_p(L.data_ptr()),
                                    ctypes.c_void_p(G.data_ptr()), ctypes.c_void_p(G.data_ptr()), 1)
    e1.record()
    torch.cuda.synchronize()
    assert st == 0, st
    d = curfp.rfp_diag_indices(n)
    G[d] -= 0.5
    err = G.abs().max().item()
    S.emit({"config": "C5-adjoint", "n": n, "k": k, "lambda": lam,
            "spftrf_backward_ms": round(e0.elapsed_time(e1), 1), "max_abs_err_vs_half_I": err,
            "peak_mem_gb": round(torch.cuda.max_memory_allocated() / 1e9, 1)})
    del L, G
    torch.cuda.empty_cache()
    assert err <= 1e-4, err
