"""Adjoint planning on CPU: the planner's Cholesky / solve / rank-k adjoint
sequences (curfp_b200/csrc/plan.cpp) bound to the CPU executor, against
closed forms evaluated in FP64, for all 8 RFP variants.  The closed forms are
themselves checked against FP64 finite differences of the forward maps, so
the cotangent convention (derivative with respect to each STORED element of
an RFP array) is pinned independently of the algebra."""
import ctypes

import numpy as np
import pytest

from conftest import VARIANTS

fp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731


def to_rfp(orc, tr, ul, Lmat):
    """RFP array (float32) of the logical lower triangle Lmat."""
    n = Lmat.shape[0]
    dense = Lmat.T if ul == 1 else Lmat
    return orc.strttf(tr, ul, n, np.ascontiguousarray(dense)).astype(np.float32)


def spd(rng, n, k=None):
    k = k or max(2, n // 2)
    X = rng.standard_normal((n, k)) / np.sqrt(k)
    return X @ X.T + np.eye(n)


def chol_adjoint_stored(L, Lbar):
    """Cotangent of the stored (lower) elements of A from that of L."""
    M = L.T @ Lbar
    Q = np.tril(M) + np.tril(M, -1).T
    Li = np.linalg.inv(L)
    S = Li.T @ Q @ Li
    G = np.tril(S)
    G[np.diag_indices_from(G)] *= 0.5
    return G


def test_chol_adjoint_formula_vs_fd():
    """<Lbar, chol(A)> differentiated w.r.t. the stored lower elements."""
    rng = np.random.default_rng(11)
    n = 9
    A = spd(rng, n)
    Lbar = np.tril(rng.standard_normal((n, n)))
    G = chol_adjoint_stored(np.linalg.cholesky(A), Lbar)
    E = np.tril(rng.standard_normal((n, n)))
    Es = E + np.tril(E, -1).T  # symmetric matrix of a stored-element change
    h = 1e-6
    f = lambda t: np.sum(Lbar * np.linalg.cholesky(A + t * Es))  # noqa: E731
    fd = (f(h) - f(-h)) / (2 * h)
    assert abs(fd - np.sum(G * E)) <= 1e-7 * max(1.0, abs(fd))


def from_rfp(orc, tr, ul, n, arf):
    """Logical lower triangle (float64) of an RFP array."""
    dense = orc.stfttr(tr, ul, n, np.asarray(arf, np.float64))
    return np.tril(dense.T if ul == 1 else dense)


def run_adjoint(orc, hostsim, tr, ul, L, Lbar):
    n = L.shape[0]
    G = to_rfp(orc, tr, ul, Lbar)
    calls = ctypes.c_long(0)
    assert hostsim.hs_spftrf_backward(tr, 1 - ul, n, fp(to_rfp(orc, tr, ul, L)), fp(G), 0,
                                      ctypes.byref(calls)) == 0
    return from_rfp(orc, tr, ul, n, G), calls.value


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 17, 64, 65, 130, 257])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_spftrf_backward_host(orc, hostsim, n, tr, ul):
    """The blocked in-place RFP adjoint (tiles of 64, panel steps between
    them) against the closed form."""
    rng = np.random.default_rng(1000 + 8 * n + 2 * tr + ul)
    L = np.linalg.cholesky(spd(rng, n)).astype(np.float32).astype(np.float64)
    Lbar = np.tril(rng.standard_normal((n, n))).astype(np.float32).astype(np.float64)
    G, _ = run_adjoint(orc, hostsim, tr, ul, L, Lbar)
    Ge = chol_adjoint_stored(L, Lbar)
    assert np.linalg.norm(G - Ge) <= 2e-5 * np.linalg.norm(Ge)


@pytest.mark.parametrize("tr,ul", [(0, 0), (1, 1), (0, 1), (1, 0)])
def test_spftrf_backward_host_recursive(orc, hostsim, tr, ul):
    """n well above the tile: several levels of panel steps, each with its
    solve and masked two-product update."""
    n = 600
    rng = np.random.default_rng(5 + tr + ul)
    L = np.linalg.cholesky(spd(rng, n)).astype(np.float32).astype(np.float64)
    Lbar = np.tril(rng.standard_normal((n, n))).astype(np.float32).astype(np.float64)
    G, calls = run_adjoint(orc, hostsim, tr, ul, L, Lbar)
    Ge = chol_adjoint_stored(L, Lbar)
    assert calls > 0
    assert np.linalg.norm(G - Ge) <= 2e-5 * np.linalg.norm(Ge)

def test_ssfrk_adjoint_formula_vs_fd(orc):
    """<Cbar, ssfrk(A)> over stored elements, differentiated w.r.t. A."""
    rng = np.random.default_rng(3)
    n, k, alpha = 7, 3, 0.7
    for tr, ul in VARIANTS:
        A = rng.standard_normal((n, k))
        Cbar = rng.standard_normal(n * (n + 1) // 2)
        Cl = orc.rfp_to_factor(tr, ul, n, Cbar)
        Ge = alpha * (Cl + Cl.T) @ A
        E = rng.standard_normal((n, k))
        h = 1e-6

        def f(t):
            At = A + t * E
            C = orc.ssfrk(tr, ul, 0, n, k, alpha, At.T.copy().ravel(), n, 0.0,
                          np.zeros(n * (n + 1) // 2))
            return float(Cbar @ C)
        fd = (f(h) - f(-h)) / (2 * h)
        assert abs(fd - np.sum(Ge * E)) <= 1e-7 * max(1.0, abs(fd))


@pytest.mark.parametrize("n,k", [(1, 1), (5, 3), (17, 4), (65, 33), (130, 20)])
@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_ssfrk_backward_host(orc, hostsim, n, k, trans, tr, ul):
    rng = np.random.default_rng(77 + n + k + trans + 2 * tr + ul)
    alpha = 0.625
    opA = rng.standard_normal((n, k)).astype(np.float32)
    Cbar = rng.standard_normal(n * (n + 1) // 2).astype(np.float32)
    # trans = N: A is n x k column-major (lda = n); trans = T: A is k x n
    # column-major (lda = k), i.e. opA row-major.
    A = np.asfortranarray(opA) if trans == 0 else np.ascontiguousarray(opA)
    Abar = np.zeros_like(A)
    lda = n if trans == 0 else k
    assert hostsim.hs_ssfrk_backward(tr, 1 - ul, trans, n, k, ctypes.c_float(alpha), fp(A),
                                     lda, fp(Cbar), fp(Abar), lda) == 0
    Cl = orc.rfp_to_factor(tr, ul, n, Cbar.astype(np.float64))
    Ge = alpha * (Cl + Cl.T) @ opA.astype(np.float64)
    assert np.linalg.norm(Abar - Ge) <= 1e-6 * np.linalg.norm(Ge) + 1e-30


def solve_adjoint(L, X, Xbar):
    A = L @ L.T
    Bbar = np.linalg.solve(A, Xbar)
    Lbar = -np.tril(Bbar @ (L.T @ X).T + X @ (L.T @ Bbar).T)
    return Bbar, Lbar


def test_solve_adjoint_formula_vs_fd():
    """<Xbar, (L L^T)^-1 B> differentiated w.r.t. B and the stored L."""
    rng = np.random.default_rng(19)
    n, m = 8, 3
    L = np.linalg.cholesky(spd(rng, n))
    B = rng.standard_normal((n, m))
    Xbar = rng.standard_normal((n, m))
    X = np.linalg.solve(L @ L.T, B)
    Bbar, Lbar = solve_adjoint(L, X, Xbar)
    E = np.tril(rng.standard_normal((n, n)))
    Eb = rng.standard_normal((n, m))
    h = 1e-6
    f = lambda t: np.sum(Xbar * np.linalg.solve((L + t * E) @ (L + t * E).T, B + t * Eb))  # noqa: E731
    fd = (f(h) - f(-h)) / (2 * h)
    assert abs(fd - np.sum(Lbar * E) - np.sum(Bbar * Eb)) <= 1e-7 * max(1.0, abs(fd))


@pytest.mark.parametrize("n,m", [(1, 1), (4, 2), (17, 1), (65, 3), (130, 7), (257, 2)])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_spftrs_backward_host(orc, hostsim, n, m, tr, ul):
    rng = np.random.default_rng(400 + n + m + 2 * tr + ul)
    L = np.linalg.cholesky(spd(rng, n)).astype(np.float32).astype(np.float64)
    X = rng.standard_normal((n, m)).astype(np.float32)
    Xbar = rng.standard_normal((n, m)).astype(np.float32)
    Xf, Xbf = np.asfortranarray(X), np.asfortranarray(Xbar)
    Bbar = np.zeros((n, m), np.float32, order="F")
    Lbar = np.zeros(n * (n + 1) // 2, np.float32)
    assert hostsim.hs_spftrs_backward(tr, 1 - ul, n, m, fp(to_rfp(orc, tr, ul, L)), fp(Xf),
                                      fp(Xbf), fp(Bbar), fp(Lbar)) == 0
    Be, Le = solve_adjoint(L, X.astype(np.float64), Xbar.astype(np.float64))
    assert np.linalg.norm(Bbar - Be) <= 1e-5 * np.linalg.norm(Be)
    Lg = orc.rfp_to_factor(tr, ul, n, Lbar.astype(np.float64))
    assert np.linalg.norm(Lg - Le) <= 1e-5 * np.linalg.norm(Le)


@pytest.mark.parametrize("n,m", [(3, 2), (65, 5), (257, 3)])
@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_rfp_trsm_host(orc, hostsim, n, m, trans, tr, ul):
    rng = np.random.default_rng(n + m + trans + 2 * tr + ul)
    L = np.linalg.cholesky(spd(rng, n)).astype(np.float32).astype(np.float64)
    B = rng.standard_normal((n, m)).astype(np.float32)
    Bf = np.asfortranarray(B)
    assert hostsim.hs_rfp_trsm(tr, 1 - ul, n, fp(to_rfp(orc, tr, ul, L)), trans, fp(Bf), m,
                               ctypes.c_float(-0.5)) == 0
    Xe = np.linalg.solve(L.T if trans else L, -0.5 * B.astype(np.float64))
    assert np.linalg.norm(Bf - Xe) <= 1e-5 * np.linalg.norm(Xe)
