"""CPU baseline: the reference's pipeline on the host cores.

TEST / BENCHMARK INFRASTRUCTURE ONLY.  The reference (andersx/curfp) runs
LAPACK's RFP algorithm (its sources call themselves direct translations of
LAPACK ssfrk.f / spftrf.f / spftrs.f, e.g. src/curfp_spftrf.cpp:1-12) through
cuBLAS/cuSOLVER; on the CPU the same algorithm is LAPACK's own RFP routines.
This module runs that pipeline -- ssfrk -> add shift to the diagonal ->
spftrf -> spftrs -- exactly as the reference's CPU oracle test does
(python_tests/test_vs_lapack.py:32-55,77-90), on scipy's LAPACK (OpenBLAS,
all threads of the process).
"""
from __future__ import annotations

import os
import time

import numpy as np
from scipy.linalg import lapack as la


def threads() -> int:
    try:
        from threadpoolctl import threadpool_info
        for info in threadpool_info():
            if info.get("internal_api") == "openblas":
                return int(info.get("num_threads", os.cpu_count() or 1))
    except Exception:
        pass
    return os.cpu_count() or 1


def diag_indices(n: int, transr: str, uplo: str) -> np.ndarray:
    from .oracle import diag_indices as di
    return di(0 if transr == "N" else 1, 0 if uplo == "L" else 1, n)


def cholesky_solve(A_nk: np.ndarray, B_n_nrhs: np.ndarray, shift: float,
                   transr: str = "T", uplo: str = "U") -> dict:
    """Time ssfrk + diagonal shift + spftrf + spftrs on the host.

    A_nk: (n, k) float32 row-major; B: (n, nrhs) float32.  Returns seconds per
    phase and the solution."""
    n, k = A_nk.shape
    Af = np.asfortranarray(A_nk, dtype=np.float32)
    t0 = time.perf_counter()
    C = la.ssfrk(n, k, 1.0, Af, 0.0, np.zeros(n * (n + 1) // 2, np.float32),
                 transr=transr, uplo=uplo, trans="N")
    t1 = time.perf_counter()
    C[diag_indices(n, transr, uplo)] += np.float32(shift)
    t2 = time.perf_counter()
    F, info = la.spftrf(n, C, transr=transr, uplo=uplo)
    t3 = time.perf_counter()
    X, info2 = la.spftrs(n, F, np.asfortranarray(B_n_nrhs, dtype=np.float32),
                         transr=transr, uplo=uplo)
    t4 = time.perf_counter()
    if info != 0 or info2 != 0:
        raise RuntimeError(f"LAPACK failed: spftrf info={info} spftrs info={info2}")
    return {"ssfrk": t1 - t0, "shift": t2 - t1, "spftrf": t3 - t2, "spftrs": t4 - t3,
            "X": X, "F": F}
