"""The oracle (plain-C restatement of the reference's table-driven algorithm)
against LAPACK golden vectors and the reference's known-answer tests."""
import numpy as np
import pytest

from conftest import VARIANTS

NS = [1, 2, 3, 4, 5, 6, 7, 8, 9, 15, 16, 17, 32, 33, 64, 65, 97]
TAG = {0: "N", 1: "T"}
UTAG = {0: "L", 1: "U"}


def key(n, tr, ul):
    return f"{n}_{TAG[tr]}{UTAG[ul]}"


@pytest.mark.parametrize("n", NS)
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_oracle_pack_and_diag(golden, orc, n, tr, ul):
    S = golden[f"S_{n}"]
    arf = orc.strttf(tr, ul, n, S)
    assert np.array_equal(arf, golden[f"strttf_{key(n, tr, ul)}"])
    back = orc.stfttr(tr, ul, n, arf)
    mask = np.triu(np.ones((n, n), bool)) if ul else np.tril(np.ones((n, n), bool))
    assert np.array_equal(back[mask], S[mask])
    assert np.array_equal(orc.diag_indices(tr, ul, n), golden[f"diag_{key(n, tr, ul)}"])


@pytest.mark.parametrize("n", NS)
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_oracle_pipeline(golden, orc, n, tr, ul):
    k = max(1, n // 2)
    A = golden[f"A_{n}"]
    B = golden[f"B_{n}"]
    kk = key(n, tr, ul)
    C = orc.ssfrk(tr, ul, 0, n, k, 1.0, A.T.ravel(), n, 0.0, np.zeros(n * (n + 1) // 2))
    np.testing.assert_allclose(C, golden[f"ssfrk_{kk}"], rtol=0, atol=1e-12)
    C[golden[f"diag_{kk}"]] += 1.0
    F, info = orc.spftrf(tr, ul, n, C)
    assert info == 0
    np.testing.assert_allclose(F, golden[f"spftrf_{kk}"], rtol=0, atol=1e-12)
    X = orc.spftrs(tr, ul, n, 3, F, B.T.ravel(), n).reshape(3, n).T
    np.testing.assert_allclose(X, golden[f"spftrs_{kk}"], rtol=0, atol=1e-10)
    Ai, rc = orc.spftri(tr, ul, n, F)
    assert rc == 0
    np.testing.assert_allclose(Ai, golden[f"spftri_{kk}"], rtol=0, atol=1e-10)


def test_oracle_kats(golden, orc):
    F, info = orc.spftrf(0, 0, 2, golden["kat_n2_NL_in"])
    assert info == 0
    np.testing.assert_allclose(F, golden["kat_n2_NL_out"], atol=1e-14)
    F, info = orc.spftrf(0, 0, 3, golden["kat_n3_NL_in"])
    assert info == 0
    np.testing.assert_allclose(F, golden["kat_n3_NL_out"], atol=1e-14)
    C = orc.ssfrk(0, 0, 0, 2, 1, 2.0, golden["kat_frk_n2_A"], 2, 0.5, golden["kat_frk_n2_C"])
    np.testing.assert_allclose(C, golden["kat_frk_n2_out"], atol=1e-14)
    # n=1: sqrt on every variant (reference python_tests/test_spftrf.py:19-39)
    for tr, ul in VARIANTS:
        F, info = orc.spftrf(tr, ul, 1, np.array([7.0]))
        assert info == 0 and abs(F[0] - np.sqrt(7.0)) < 1e-15


@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_oracle_quick_returns(orc, tr, ul):
    n = 5
    C0 = np.arange(n * (n + 1) // 2, dtype=np.float64)
    # alpha = 0, beta = 1 -> untouched; alpha = beta = 0 -> zero (A unused)
    assert np.array_equal(orc.ssfrk(tr, ul, 0, n, 3, 0.0, None, n, 1.0, C0), C0)
    assert not orc.ssfrk(tr, ul, 0, n, 3, 0.0, None, n, 0.0, C0).any()


@pytest.mark.parametrize("tr,ul", VARIANTS)
@pytest.mark.parametrize("n,bad", [(6, 2), (6, 5), (7, 1), (7, 6)])
def test_oracle_info(orc, tr, ul, n, bad):
    """Non-SPD: info = order of the first failing leading minor, offset into
    the second block (reference src/curfp_spftrf.cpp:259,282)."""
    M = np.eye(n) * 2.0
    M[bad - 1, bad - 1] = -1.0
    arf = orc.strttf(tr, ul, n, M)
    _, info = orc.spftrf(tr, ul, n, arf)
    assert info == bad
