"""Index arithmetic of two kernels, checked on the host (no GPU):

* the single-read symmetric matrix-vector product (ssfmv / dsfmv): its CTAs
  visit every 64 x 64 tile of the lower triangle exactly once, and every
  row / column partial sum lands in its own slot inside the partial-sum
  buffer (curfp_b200/csrc/symv_layout.h);
* the routing of contractions to the few-column kernels
  (curfp_b200/csrc/gemm_route.h): which products qualify, when the product
  is transposed, which kernel and instantiation take it."""
import ctypes

import numpy as np
import pytest


def layout(hs, n):
    out = np.zeros(7, np.int64)
    assert hs.hs_symv_layout(n, out.ctypes.data_as(ctypes.c_void_p)) == 0
    return out


@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 127, 1000, 1023, 1024, 1025, 4097, 16384,
                               20001, 32767, 32768, 65536, 131072])
def test_symv_tiles_visited_once(hostsim, n):
    ctas, visited, dup, row_over, col_over, col_dup, empty = layout(hostsim, n)
    T = (n + 63) // 64
    assert visited == T * (T + 1) // 2
    assert dup == 0 and row_over == 0 and col_over == 0 and col_dup == 0
    assert empty == 0
    # one CTA per strip of 16 tiles: sum over tile rows of ceil((I + 1) / 16)
    assert ctas == sum((i // 16) + 1 for i in range(T))


def route(hs, m, n, k, k2=0, a_tri=0, b_tri=0, c_lower=0, inplace=0, a_rs=1, a_cs=None):
    out = (ctypes.c_int * 7)()
    if a_cs is None:
        a_cs = m  # column-major A
    assert hs.hs_skinny_route(m, n, k, k2, a_tri, b_tri, c_lower, inplace,
                              ctypes.c_int64(a_rs), ctypes.c_int64(a_cs), out) == 0
    return list(out)


@pytest.mark.parametrize("ncols,inst", [(1, 1), (2, 2), (3, 4), (4, 4), (5, 8), (8, 8)])
def test_skinny_route_few_columns(hostsim, ncols, inst):
    use, transpose, rows, got_inst, m, n, k = route(hostsim, 16384, ncols, 16384)
    assert (use, transpose, rows, got_inst) == (1, 0, 1, inst)
    assert (m, n, k) == (16384, ncols, 16384)
    # A with unit-stride columns (row-major A): the column kernel
    use, transpose, rows, got_inst, *_ = route(hostsim, 16384, ncols, 16384, a_rs=16384, a_cs=1)
    assert (use, transpose, rows, got_inst) == (1, 0, 0, inst)


def test_skinny_route_transposed(hostsim):
    """m <= 8 < n: computed as C^T = B^T A^T; the routed A is B^T (n x k),
    whose row index is B's column index (stride k for column-major B)."""
    use, transpose, rows, inst, m, n, k = route(hostsim, 3, 20000, 4096)
    assert (use, transpose, inst, m, n, k) == (1, 1, 4, 20000, 3, 4096)
    assert rows == 0  # B^T (n x k) is unit-stride along k


@pytest.mark.parametrize("kw", [dict(k2=5), dict(a_tri=1), dict(b_tri=2), dict(c_lower=1),
                                dict(inplace=1), dict(a_rs=7, a_cs=16384 * 7)])
def test_skinny_route_declines(hostsim, kw):
    assert route(hostsim, 16384, 1, 16384, **kw)[0] == 0


def test_skinny_route_small_or_wide(hostsim):
    assert route(hostsim, 1000, 1, 1000)[0] == 0        # < 2^20 elements of A
    assert route(hostsim, 16384, 9, 16384)[0] == 0      # 9 columns: the tiled kernel
    assert route(hostsim, 1024, 1, 1024)[0] == 1        # exactly 2^20
    assert route(hostsim, 16384, 1, 0)[0] == 0          # k = 0: beta C only
