"""slansf / spfcon / spftrf_rcond on the GPU, all 8 variants.

slansf against FP64 numpy norms of the dense symmetric matrix (MAX exact,
ONE and FRO within 1e-6 relative: the library sums in FP64).  spfcon
against scipy's LAPACK spocon within the factor 3 of the reference's own
test (python_tests/test_spfcon.py:29-105) and against the CPU restatement of
the estimator (oracle/condest.py) driven by an FP64 solve with the same
factor, within 1e-4 relative (same iteration path; FP32 vs FP64 solves)."""
import numpy as np
import pytest
import scipy.linalg
import torch
from scipy.linalg import lapack

from conftest import VARIANTS
from helpers import TR, UL, dev, host
from oracle import condest

NS = [1, 2, 3, 4, 5, 8, 16, 63, 64, 65, 255, 256, 1000, 1023]


def make_sym(n, rng):
    B = rng.standard_normal((n, n)).astype(np.float32)
    return (B @ B.T + n * np.eye(n, dtype=np.float32)).astype(np.float32)


def to_rfp(curfp, A, tr, ul):
    tri = np.triu(A) if ul else np.tril(A)
    return curfp.strttf(dev(tri), transr=TR[tr], uplo=UL[ul])


@pytest.mark.gpu
@pytest.mark.parametrize("n", NS)
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_slansf(curfp, n, tr, ul):
    rng = np.random.default_rng(100 + n)
    A = make_sym(n, rng)
    A[rng.integers(0, n), rng.integers(0, n)] *= -1  # a negative element somewhere
    A = np.triu(A) + np.triu(A, 1).T if ul else np.tril(A) + np.tril(A, -1).T
    arf = to_rfp(curfp, A, tr, ul)
    A64 = A.astype(np.float64)
    kw = dict(transr=TR[tr], uplo=UL[ul])
    assert curfp.slansf(arf, "M", **kw) == float(np.abs(A).max())
    one = float(np.abs(A64).sum(axis=0).max())
    assert abs(curfp.slansf(arf, "1", **kw) - one) <= 1e-6 * one
    assert curfp.slansf(arf, "I", **kw) == curfp.slansf(arf, "O", **kw)
    fro = float(np.linalg.norm(A64))
    assert abs(curfp.slansf(arf, "F", **kw) - fro) <= 1e-6 * fro


@pytest.mark.gpu
def test_slansf_edges(curfp):
    assert curfp.slansf(torch.empty(0, device="cuda"), "1", n=0) == 0.0
    arf = torch.tensor([-7.5], device="cuda")
    for s in ("M", "1", "F"):
        assert curfp.slansf(arf, s) == 7.5
    with pytest.raises(ValueError):
        curfp.slansf(arf, "X")
    h = curfp.Handle()
    with pytest.raises(RuntimeError, match="status=3"):
        curfp.slansf_raw(h, 7, curfp.OP_T, curfp.FILL_UPPER, 1, arf)
    assert curfp.slansf_raw(h, curfp.NORM_MAX, curfp.OP_T, curfp.FILL_UPPER, 1, arf) == 7.5
    h.close()


def make_spd(n, rng, cond):
    if n == 1:
        return np.array([[1.0]], dtype=np.float32)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    return ((Q * np.linspace(1.0, cond, n)) @ Q.T).astype(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("cond", [10.0, 1e4])
@pytest.mark.parametrize("n", [1, 2, 3, 8, 32, 64, 128, 256, 600])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_spfcon(curfp, orc, n, cond, tr, ul):
    rng = np.random.default_rng(42 + n)
    A = make_spd(n, rng, cond)
    A = np.triu(A) + np.triu(A, 1).T if ul else np.tril(A) + np.tril(A, -1).T
    kw = dict(transr=TR[tr], uplo=UL[ul])
    arf = to_rfp(curfp, A, tr, ul)
    anorm = curfp.slansf(arf, "1", **kw)
    assert abs(anorm - np.linalg.norm(A.astype(np.float64), 1)) <= 1e-6 * anorm
    assert curfp.spftrf(arf, **kw) == 0
    got = curfp.spfcon(arf, anorm, **kw)
    U = scipy.linalg.cholesky(A.astype(np.float64), lower=False)
    want, info = lapack.dpocon(U, anorm)
    assert info == 0
    assert 1 / 3 <= got / want <= 3, (got, want)
    L = orc.rfp_to_factor(tr, ul, n, host(arf).astype(np.float64))
    port = condest.spfcon(condest.dense_factor_solver(L), n, anorm)
    assert abs(got - port) <= 1e-4 * port, (got, port)


@pytest.mark.gpu
def test_spfcon_edges_and_rcond(curfp):
    arf = torch.tensor([5.0], device="cuda")
    curfp.spftrf(arf)
    assert abs(curfp.spfcon(arf, 5.0) - 1.0) < 1e-6
    assert curfp.spfcon(arf, 0.0) == 0.0
    rng = np.random.default_rng(7)
    A = make_spd(300, rng, 50.0)
    arf = to_rfp(curfp, A, 1, 1)
    arf2 = arf.clone()
    anorm = curfp.slansf(arf, "1")
    curfp.spftrf(arf)
    r1 = curfp.spfcon(arf, anorm)
    h = curfp.Handle()
    r2 = curfp.spfcon_raw(h, curfp.OP_T, curfp.FILL_UPPER, 300, arf, anorm)
    h.close()
    assert r1 == r2
    assert curfp.spftrf_rcond(arf2) == r1
    torch.testing.assert_close(arf2, arf, rtol=0, atol=0)
    bad = to_rfp(curfp, -np.eye(4, dtype=np.float32), 1, 1)
    with pytest.raises(torch.linalg.LinAlgError):
        curfp.spftrf_rcond(bad.clone())
    assert curfp.spftrf_rcond(bad.clone(), check=False) == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("tr,ul", [(1, 1), (0, 0)])
def test_slansf_large(curfp, tr, ul):
    """n = 20001 (odd, 2e8 elements): FP64 torch norms of the dense matrix."""
    n = 20001
    g = torch.Generator(device="cuda").manual_seed(5)
    M = torch.randn(n, n, device="cuda", generator=g)
    arf = curfp.strttf(M, transr=TR[tr], uplo=UL[ul])
    T = (M.triu() if ul else M.tril()).double()
    S = T + (T.triu(1).T if ul else T.tril(-1).T)
    kw = dict(transr=TR[tr], uplo=UL[ul])
    assert curfp.slansf(arf, "M", **kw) == float(S.abs().max())
    one = float(S.abs().sum(dim=0).max())
    assert abs(curfp.slansf(arf, "1", **kw) - one) <= 1e-6 * one
    fro = float(torch.linalg.norm(S))
    assert abs(curfp.slansf(arf, "F", **kw) - fro) <= 1e-6 * fro
