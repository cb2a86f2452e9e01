"""Host logic of the library on CPU: the planner (curfp_b200/csrc/plan.cpp)
bound to a CPU executor, against the oracle, for all 8 variants and sizes that
exercise the recursion (> 64) and odd splits.  Also the view geometry against
the LAPACK strttf golden vectors."""
import ctypes

import numpy as np
import pytest

from conftest import VARIANTS

fp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731


def geometry(hs, n, tr, ul):
    out = np.zeros(11, np.int64)
    hs.hs_geometry(n, tr, 1 - ul, out.ctypes.data_as(ctypes.c_void_p))
    return out


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 16, 17, 64, 65, 97])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_view_geometry_vs_lapack(golden, hostsim, n, tr, ul):
    """arf[off + p*rs + q*cs] of each block == logical S[p, q] (p >= q)."""
    g = geometry(hostsim, n, tr, ul)
    n1 = g[0]
    arf = golden[f"strttf_{n}_{'NT'[tr]}{'LU'[ul]}"]
    S = golden[f"S_{n}"]
    seen = set()
    for p in range(n):
        for q in range(p + 1):
            if q < n1 and p < n1:
                o, rs, cs = g[2:5]; a = o + p * rs + q * cs
            elif q < n1:
                o, rs, cs = g[5:8]; a = o + (p - n1) * rs + q * cs
            else:
                o, rs, cs = g[8:11]; a = o + (p - n1) * rs + (q - n1) * cs
            assert arf[a] == S[p, q]
            seen.add(int(a))
    assert len(seen) == n * (n + 1) // 2


@pytest.mark.parametrize("n", [1, 2, 3, 7, 64, 65, 128, 129, 200, 257])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_planner_pipeline(orc, hostsim, n, tr, ul):
    rng = np.random.default_rng(7 * n + 3 * tr + ul)
    k = max(1, n // 3)
    A = (rng.standard_normal((n, k)) / np.sqrt(k)).astype(np.float32)
    C = np.zeros(n * (n + 1) // 2, np.float32)
    assert hostsim.hs_ssfrk(tr, 1 - ul, 1, n, k, ctypes.c_float(1.0), fp(A), k,
                            ctypes.c_float(0.0), fp(C), None) == 0
    Co = orc.ssfrk(tr, ul, 1, n, k, 1.0, A.astype(np.float64), k, 0.0,
                   np.zeros(n * (n + 1) // 2))
    np.testing.assert_allclose(C, Co, atol=2e-6)
    di = orc.diag_indices(tr, ul, n)
    C[di] += 1.0
    Co[di] += 1.0
    F = C.copy()
    info = ctypes.c_int(-1)
    assert hostsim.hs_spftrf(tr, 1 - ul, n, fp(F), ctypes.byref(info)) == 0
    Fo, info_o = orc.spftrf(tr, ul, n, Co)
    assert info.value == info_o == 0
    np.testing.assert_allclose(F, Fo, atol=5e-6)
    B = rng.standard_normal((4, n)).astype(np.float32)
    X = B.copy()
    assert hostsim.hs_spftrs(tr, 1 - ul, n, 4, fp(F), fp(X), n) == 0
    Xo = orc.spftrs(tr, ul, n, 4, Fo, B.astype(np.float64).ravel(), n)
    np.testing.assert_allclose(X.ravel(), Xo, atol=5e-5 * max(1, np.abs(Xo).max()))
    Inv = F.copy()
    assert hostsim.hs_spftri(tr, 1 - ul, n, fp(Inv)) == 0
    Io, rc = orc.spftri(tr, ul, n, Fo)
    np.testing.assert_allclose(Inv, Io, atol=5e-5 * max(1, np.abs(Io).max()))


@pytest.mark.parametrize("n", [5, 70, 131])
@pytest.mark.parametrize("tr,ul", VARIANTS)
@pytest.mark.parametrize("trans", [0, 1])
def test_planner_ssfr2k(orc, hostsim, n, tr, ul, trans):
    rng = np.random.default_rng(n + 10 * trans)
    k = 9
    shape = (k, n) if trans == 0 else (n, k)  # row-major storage of col-major op
    A = rng.standard_normal(shape).astype(np.float32)
    B = rng.standard_normal(shape).astype(np.float32)
    lda = n if trans == 0 else k
    C = rng.standard_normal(n * (n + 1) // 2).astype(np.float32)
    Co = orc.ssfr2k(tr, ul, trans, n, k, 0.5, A, lda, B, lda, -1.5, C)
    assert hostsim.hs_ssfr2k(tr, 1 - ul, trans, n, k, ctypes.c_float(0.5), fp(A), lda,
                             fp(B), lda, ctypes.c_float(-1.5), fp(C)) == 0
    np.testing.assert_allclose(C, Co, atol=1e-4)


@pytest.mark.parametrize("tr,ul", VARIANTS)
@pytest.mark.parametrize("n,bad", [(10, 3), (10, 8), (150, 1), (150, 70), (150, 149)])
def test_planner_info(orc, hostsim, tr, ul, n, bad):
    M = np.eye(n) * 2.0
    M[bad - 1, bad - 1] = -1.0
    arf = orc.strttf(tr, ul, n, M).astype(np.float32)
    info = ctypes.c_int(-1)
    assert hostsim.hs_spftrf(tr, 1 - ul, n, fp(arf), ctypes.byref(info)) == 0
    assert info.value == bad


@pytest.mark.parametrize("n,m", [(1, 3), (2, 1), (7, 5), (64, 3), (65, 8), (130, 1)])
@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_planner_ssfmm(orc, hostsim, n, m, side, tr, ul):
    """rfp_symm (ssfmm / ssfmv planning, strict-upper mask on the transposed
    triangles) against the dense symmetric product: side 0 C = a A B + b C
    (B n x m), side 1 C = a B A + b C (B m x n); column-major."""
    rng = np.random.default_rng(11 * n + m + side)
    nt = n * (n + 1) // 2
    arf = rng.standard_normal(nt).astype(np.float32)
    A = orc.rfp_to_dense_sym(tr, ul, n, arf.astype(np.float64))
    rows, cols = (n, m) if side == 0 else (m, n)
    B = np.asfortranarray(rng.standard_normal((rows, cols)).astype(np.float32))
    C = np.asfortranarray(rng.standard_normal((rows, cols)).astype(np.float32))
    want = 0.5 * (A @ B if side == 0 else B @ A) - 2.0 * C.astype(np.float64)
    assert hostsim.hs_ssfmm(tr, 1 - ul, side, rows, cols, ctypes.c_float(0.5), fp(arf), fp(B),
                            rows, ctypes.c_float(-2.0), fp(C), rows) == 0
    np.testing.assert_allclose(C, want, rtol=1e-5, atol=1e-5)
    # alpha = 0: C := beta C without reading A or B
    C0 = C.copy()
    bad = np.full(nt, np.nan, np.float32)
    assert hostsim.hs_ssfmm(tr, 1 - ul, side, rows, cols, ctypes.c_float(0.0), fp(bad),
                            fp(np.full_like(B, np.nan)), rows, ctypes.c_float(3.0), fp(C),
                            rows) == 0
    np.testing.assert_array_equal(C, 3.0 * C0)
