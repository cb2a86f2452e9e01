"""The CPU restatement of the condition estimator (oracle/condest.py) against
LAPACK's spocon (scipy) on SPD matrices like the reference's spfcon tests
(python_tests/test_spfcon.py:29-41: eigenvalues spaced from 1 to cond in a
random orthogonal basis), within the factor 3 that test allows, plus the
n = 1 and anorm = 0 cases."""
import numpy as np
import pytest
import scipy.linalg
from scipy.linalg import lapack

from oracle import condest


def make_spd(n, rng, cond):
    if n == 1:
        return np.array([[1.0]])
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    return (Q * np.linspace(1.0, cond, n)) @ Q.T


@pytest.mark.parametrize("cond", [10.0, 1e4])
@pytest.mark.parametrize("n", [2, 3, 4, 8, 16, 32, 64, 128, 256])
def test_oracle_vs_spocon(n, cond):
    rng = np.random.default_rng(42 + n)
    A = make_spd(n, rng, cond).astype(np.float32).astype(np.float64)
    U = scipy.linalg.cholesky(A, lower=False)
    anorm = float(np.linalg.norm(A, 1))
    want, info = lapack.dpocon(U, anorm)
    assert info == 0
    got = condest.spfcon(condest.dense_factor_solver(U.T), n, anorm)
    assert 1 / 3 <= got / want <= 3, (got, want)
    # the estimate never exceeds the true rcond (it underestimates ||A^-1||_1)
    true = 1.0 / (anorm * np.linalg.norm(np.linalg.inv(A), 1))
    assert got >= true * (1 - 1e-12)


def test_oracle_edge_cases():
    assert condest.spfcon(lambda x: x / 5.0, 1, 5.0) == pytest.approx(1.0)
    assert condest.spfcon(lambda x: x, 4, 0.0) == 0.0
    assert condest.spfcon(lambda x: x, 0, 1.0) == 0.0
