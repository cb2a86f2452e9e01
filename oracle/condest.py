"""CPU restatement of the reference's 1-norm condition estimator.

TEST INFRASTRUCTURE ONLY (the checker of curfpSpfcon; never on the product
path).  Follows src/curfp_spfcon.cu:140-257 of the reference, its port of
LAPACK SLACN2 (Hager-Higham) for an SPD matrix, where A^-T = A^-1 so every
reverse-communication request is one solve:

  x = 1/n; x = A^-1 x; est = |x|_1; (n == 1: done)
  x = sign(x) (saved as isgn); x = A^-1 x; j = argmax |x|; iter = 2
  loop: x = A^-1 e_j; est = |x|_1
        if sign(x) repeats isgn: go to final
        x = sign(x) (saved); x = A^-1 x; j' = argmax |x|
        if |x_j| != |x_j'| and iter < 5: j = j'; iter += 1; repeat loop
  final: x_i = (-1)^i (1 + i/(n-1)); x = A^-1 x; est = max(est, 2|x|_1 / (3n))
  rcond = (1/est) / anorm   (0 when n == 0, anorm == 0 or est == 0)

As in the reference there is no cycling test (SLACN2's "est <= estold"
exit).  The repeated-sign test treats zeros as matching (the reference
compares dot(isgn, x) with sum |x|).  Argmax ties go to the smallest index
(BLAS isamax).  Pinned in tests/test_condest_oracle.py against scipy's
LAPACK spocon on the reference test's matrices.
"""
from __future__ import annotations

from typing import Callable

import numpy as np


def _sign(x: np.ndarray) -> np.ndarray:
    return np.where(x >= 0, 1.0, -1.0)


def spfcon(solve: Callable[[np.ndarray], np.ndarray], n: int, anorm: float,
           itmax: int = 5) -> float:
    """rcond estimate; solve(x) returns A^-1 x (float64 vectors)."""
    if n == 0 or anorm == 0.0:
        return 0.0
    x = solve(np.full(n, 1.0 / n))
    est = float(np.abs(x).sum())
    if n > 1:
        isgn = _sign(x)
        x = solve(isgn.copy())
        j = int(np.argmax(np.abs(x)))
        it = 2
        while True:
            e = np.zeros(n)
            e[j] = 1.0
            x = solve(e)
            est = float(np.abs(x).sum())
            s = _sign(x)
            if not np.any((x != 0) & (s != isgn)):
                break
            isgn = s
            x = solve(s.copy())
            jn = int(np.argmax(np.abs(x)))
            if abs(x[j]) != abs(x[jn]) and it < itmax:
                j = jn
                it += 1
                continue
            break
        i = np.arange(n)
        alt = np.where(i % 2 == 0, 1.0, -1.0) * (1.0 + i / (n - 1))
        x = solve(alt)
        est = max(est, 2.0 * float(np.abs(x).sum()) / (3.0 * n))
    return (1.0 / est) / anorm if est > 0 else 0.0


def dense_factor_solver(L: np.ndarray) -> Callable[[np.ndarray], np.ndarray]:
    """x -> (L L^T)^-1 x in FP64 for a lower-triangular factor L."""
    from scipy.linalg import solve_triangular
    L = np.asarray(L, np.float64)

    def solve(b: np.ndarray) -> np.ndarray:
        y = solve_triangular(L, b, lower=True)
        return solve_triangular(L.T, y, lower=False)
    return solve
