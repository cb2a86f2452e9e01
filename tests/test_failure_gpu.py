"""Failure detection of the kernels' waits, tested without a GPU fault: a
wavefront solve whose first block row never runs leaves the next rows
waiting on a flag that nothing sets.  Their waits are bounded (~2 s of
globaltimer): they record error code 5, poison their own flags so that
dependents stop too, and return.  The call reports EXECUTION_FAILED with code
5 within a few seconds, and the same handle then solves correctly."""
import time

import numpy as np
import pytest
import torch


@pytest.mark.gpu
def test_wave_wait_times_out_and_context_survives(curfp, orc):
    from curfp_b200 import precision as P
    t0 = time.monotonic()
    status, code = P.diag_wait_timeout()
    elapsed = time.monotonic() - t0
    assert status == 4 and code == 5, (status, code)
    assert elapsed < 30.0
    # the context and the handle are usable afterwards
    n, k = 1000, 64
    rng = np.random.default_rng(3)
    A = (rng.standard_normal((n, k)) / np.sqrt(k)).astype(np.float32)
    C = torch.empty(n * (n + 1) // 2, device="cuda")
    curfp.ssfrk(torch.from_numpy(A).cuda(), C)
    curfp.add_to_diagonal(C, 1.0)
    C0 = C.clone()
    assert curfp.spftrf(C) == 0
    B = torch.randn(n, 3, device="cuda", dtype=torch.float32)
    X = B.clone()
    curfp.spftrs(C, X)
    S = curfp.stfttr(C0).double()
    S = S + S.triu(1).T
    r = (B.double() - S @ X.double()).abs().max() / (S.abs().sum(1).max() * X.double().abs().max())
    assert r.item() < 1e-6
