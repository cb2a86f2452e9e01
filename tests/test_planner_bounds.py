"""Every element range the planner hands to a kernel stays inside a caller
buffer or a workspace it asked for, at the large orders of the scale
workloads (n = 32767 ... 131072, RFP arrays of up to 8.6e9 elements, past
the int32 range), for all 8 variants and every RFP routine.  A dry-run
executor (tests/hostsim/exec_bounds.cpp) runs the planner without arithmetic
and checks each view's extreme addresses."""
import ctypes

import numpy as np
import pytest

from conftest import VARIANTS

OPS = {"ssfrk": 0, "spftrf": 1, "spftrs": 2, "spftri": 3, "trsm_n": 4, "trsm_t": 5, "trtri": 6,
       "adjoint": 7, "ssfr2k": 8}


def bounds(hs, op, tr, ul, n, k, math):
    out = np.zeros(3, np.int64)
    msg = ctypes.create_string_buffer(256)
    rc = hs.hs_bounds(OPS[op], tr, 1 - ul, n, k, math, out.ctypes.data_as(ctypes.c_void_p), msg)
    return rc, out, msg.value.decode()


@pytest.mark.parametrize("n,k", [(46341, 64), (65535, 2048), (65536, 256), (131071, 64),
                                 (131072, 4096)])
@pytest.mark.parametrize("tr,ul", VARIANTS)
@pytest.mark.parametrize("op", list(OPS))
def test_views_in_bounds_large_n(hostsim, op, tr, ul, n, k):
    for math in ((0, 1) if op in ("spftrf", "ssfrk", "trtri", "adjoint", "ssfr2k") else (0,)):
        rc, (calls, checks, bad), msg = bounds(hostsim, op, tr, ul, n, k, math)
        assert rc == 0, (rc, msg)
        assert calls > 0 and checks > 0
        assert bad == 0, msg


def test_bounds_checker_catches_overrun(hostsim):
    """The checker itself: spftrs of k right-hand sides into a B buffer one
    column short must be reported."""
    out = np.zeros(3, np.int64)
    msg = ctypes.create_string_buffer(256)
    rc = hostsim.hs_bounds_short_b(4096, 64, out.ctypes.data_as(ctypes.c_void_p), msg)
    assert rc == 0 and out[2] > 0, msg.value
