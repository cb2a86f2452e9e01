"""The FP64 checkers of tests/scale_lib.py on CPU: the RFP row gather
against the oracle's dense expansion, and the Woodbury (Gram-matrix) oracle
of C = A A^T + lam I -- solve, residual, norms, log-determinant, traces and
the GP NLL loss and gradients -- against dense FP64 computations and torch
autograd at small n."""
import numpy as np
import pytest
import torch

from conftest import VARIANTS
from scale_lib import GramOracle, nll_exact, rfp_offsets, solve_errors


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 8, 9, 64, 65])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_rfp_row_offsets(orc, n, tr, ul):
    nt = n * (n + 1) // 2
    arf = np.arange(nt, dtype=np.float64)
    D = orc.rfp_to_dense_sym(tr, ul, n, arf)
    rows = torch.arange(n)
    offs = rfp_offsets(tr, ul, n, rows).numpy()
    assert offs.min() >= 0 and offs.max() < nt
    np.testing.assert_array_equal(arf[offs], D)


@pytest.fixture(scope="module")
def small():
    rng = np.random.default_rng(3)
    n, k, lam = 300, 12, 1e-2
    A = torch.from_numpy((rng.standard_normal((n, k)) / np.sqrt(k)).astype(np.float32))
    C = A.double() @ A.double().T + lam * torch.eye(n, dtype=torch.float64)
    return A, lam, C, GramOracle(A, lam)


def test_gram_oracle_vs_dense(small):
    A, lam, C, orc = small
    n = C.shape[0]
    B = torch.from_numpy(np.random.default_rng(4).standard_normal((n, 5)))
    torch.testing.assert_close(orc.apply(B), C @ B, rtol=1e-12, atol=1e-12)
    X = torch.linalg.solve(C, B)
    torch.testing.assert_close(orc.solve(B), X, rtol=1e-9, atol=0)
    ev = torch.linalg.eigvalsh(C)
    assert abs(orc.norm2 - float(ev.max())) < 1e-10 * orc.norm2
    assert abs(orc.cond2 - float(ev.max() / ev.min())) < 1e-8 * orc.cond2
    assert abs(orc.logdet() - float(torch.logdet(C))) < 1e-9 * abs(orc.logdet())
    Ci = torch.linalg.inv(C)
    assert abs(orc.trace_inv() - float(torch.trace(Ci))) < 1e-9 * orc.trace_inv()
    Ad = A.double()
    assert abs(orc.trace_ata_cinv() - float(torch.trace(Ad.T @ Ci @ Ad))) < 1e-9
    torch.testing.assert_close(orc.cinv_a(), Ci @ Ad, rtol=1e-8, atol=1e-10)


def test_solve_errors_scale(small):
    """The exact solution has (numerically) zero error; x (1 + d) has residual
    d b, so backward error d |b| / (|C| |x| (1 + d) + |b|) and forward error d."""
    A, lam, C, orc = small
    n = C.shape[0]
    B = torch.from_numpy(np.random.default_rng(5).standard_normal((3, n)).astype(np.float32))
    X = torch.linalg.solve(C, B.double().T).T
    e = solve_errors(orc, B, X)
    assert e["backward"] < 1e-14 and e["forward"] < 1e-10
    d = 1e-6
    e = solve_errors(orc, B, X * (1 + d))
    bn, xn = B.double().norm(dim=1), X.norm(dim=1)
    want = float((d * bn / (orc.norm2 * xn * (1 + d) + bn)).max())
    assert abs(e["backward"] - want) < 1e-3 * want
    assert abs(e["forward"] - d) < 1e-3 * d


def test_nll_exact_vs_autograd(small):
    A, lam, C, orc = small
    n = C.shape[0]
    y = torch.from_numpy(np.random.default_rng(6).standard_normal(n).astype(np.float32))
    loss64, gx64, gs64, gv64 = nll_exact(orc, y)
    X = A.double().requires_grad_(True)
    s = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    v = torch.tensor(lam, dtype=torch.float64, requires_grad=True)
    Cd = s * X @ X.T + v * torch.eye(n, dtype=torch.float64)
    L = torch.linalg.cholesky(Cd)
    al = torch.cholesky_solve(y.double()[:, None], L)[:, 0]
    loss = 0.5 * torch.dot(y.double(), al) + torch.log(torch.diagonal(L)).sum()
    loss.backward()
    assert abs(loss64 - float(loss)) < 1e-9 * abs(float(loss))
    torch.testing.assert_close(gx64, X.grad, rtol=1e-7, atol=1e-7)
    assert abs(gs64 - float(s.grad)) < 1e-7 * abs(float(s.grad))
    assert abs(gv64 - float(v.grad)) < 1e-7 * abs(float(v.grad))
