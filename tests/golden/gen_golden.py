"""Generate tests/golden/lapack_rfp.npz: LAPACK golden vectors for the RFP path.

    python tests/golden/gen_golden.py

The reference's own tests pin curfp against LAPACK through scipy
(python_tests/test_vs_lapack.py:32-90, python_tests/test_stfttr_strttf.py:44-116)
plus hand-computed known-answer tests (python_tests/test_spftrf.py:42-128,
python_tests/test_ssfrk.py:84-111, tests/test_spftrf.cu, tests/test_ssfrk.cu).
This script records the same kind of vectors once, from scipy 1.18 LAPACK
(OpenBLAS), so tests on machines without scipy-matching builds compare
against fixed numbers:

  for every variant (transr N/T x uplo L/U) and n in N_LIST:
    strttf   : triangle of a seeded symmetric matrix -> RFP   (dtrttf)
    diag     : RFP offsets of the diagonal, read back from dtrttf of diag(1..n)
    ssfrk    : C = A A^T (A seeded n x k, float32 data)       (dsfrk)
    spftrf   : factor of C + I                                (dpftrf)
    spftrs   : X = (C + I)^{-1} B, 3 right-hand sides         (dpftrs)
    spftri   : (C + I)^{-1} in RFP                            (dpftri)
All arithmetic is FP64 on float32-representable inputs.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
from scipy.linalg import lapack as la

N_LIST = [1, 2, 3, 4, 5, 6, 7, 8, 9, 15, 16, 17, 32, 33, 64, 65, 97]
OUT = Path(__file__).resolve().parent / "lapack_rfp.npz"


def main() -> None:
    d = {}
    for n in N_LIST:
        rng = np.random.default_rng(1000 + n)
        k = max(1, n // 2)
        S = rng.standard_normal((n, n)).astype(np.float32).astype(np.float64)
        S = S + S.T
        A = (rng.standard_normal((n, k)) / np.sqrt(k)).astype(np.float32).astype(np.float64)
        B = rng.standard_normal((n, 3)).astype(np.float32).astype(np.float64)
        d[f"S_{n}"] = S
        d[f"A_{n}"] = A
        d[f"B_{n}"] = B
        for tr in "NT":
            for ul in "LU":
                key = f"{n}_{tr}{ul}"
                arf, info = la.dtrttf(S, transr=tr, uplo=ul)
                assert info == 0
                d[f"strttf_{key}"] = arf
                D = np.diag(np.arange(1, n + 1, dtype=np.float64))
                darf, _ = la.dtrttf(D, transr=tr, uplo=ul)
                pos = {int(v): i for i, v in enumerate(darf) if v != 0}
                d[f"diag_{key}"] = np.array([pos[i + 1] for i in range(n)], np.int64)
                C = la.dsfrk(n, k, 1.0, np.asfortranarray(A), 0.0,
                             np.zeros(n * (n + 1) // 2), transr=tr, uplo=ul,
                             trans="N")
                d[f"ssfrk_{key}"] = C
                Cs = C.copy()
                Cs[d[f"diag_{key}"]] += 1.0
                F, info = la.dpftrf(n, Cs, transr=tr, uplo=ul)
                assert info == 0
                d[f"spftrf_{key}"] = F
                X, info = la.dpftrs(n, F, np.asfortranarray(B), transr=tr, uplo=ul)
                assert info == 0
                d[f"spftrs_{key}"] = X
                Ainv, info = la.dpftri(n, F.copy(), transr=tr, uplo=ul)
                assert info == 0
                d[f"spftri_{key}"] = Ainv

    # Known-answer tests of the reference (values restated, not copied code).
    # n=2, transr=N, uplo=L, A=[[4,2],[2,3]]: RFP {a11, a00, a10}
    d["kat_n2_NL_in"] = np.array([3.0, 4.0, 2.0])
    d["kat_n2_NL_out"] = np.array([np.sqrt(2.0), 2.0, 1.0])
    # n=3, transr=N, uplo=L, A=[[5,1,2],[1,4,0],[2,0,6]]:
    # RFP {a00, a10, a20, a22, a11, a21}
    a = np.array([[5.0, 1, 2], [1, 4, 0], [2, 0, 6]])
    L = np.linalg.cholesky(a)
    d["kat_n3_NL_in"] = np.array([5.0, 1, 2, 6, 4, 0])
    d["kat_n3_NL_out"] = np.array([L[0, 0], L[1, 0], L[2, 0], L[2, 2], L[1, 1], L[2, 1]])
    # ssfrk n=2, transr=N, uplo=L, trans=N, k=1, alpha=2, beta=0.5,
    # a=[2,3], C=[[1,.5],[.5,4]] in RFP {c11, c00, c10}
    d["kat_frk_n2_C"] = np.array([4.0, 1.0, 0.5])
    d["kat_frk_n2_A"] = np.array([2.0, 3.0])
    d["kat_frk_n2_out"] = np.array([2 * 9 + 0.5 * 4, 2 * 4 + 0.5 * 1, 2 * 6 + 0.5 * 0.5])
    np.savez_compressed(OUT, **d)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(d)} arrays)")


if __name__ == "__main__":
    main()
