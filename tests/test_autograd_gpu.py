"""Differentiation form on the GPU: the hand-written adjoints behind
curfp_b200.autograd against FP64 finite differences and against dense
torch.linalg.cholesky autograd on the unpacked matrices.

Tolerances (relative, Frobenius norm over the whole gradient):
* per-op adjoints vs their FP64 closed forms on the same FP32 inputs: 2e-5
  (FP32 arithmetic, well-conditioned inputs);
* NLL gradient vs FP64 finite differences (n=256, k=32): 1e-4;
* NLL gradient vs dense FP64 torch autograd (n=8192, d=256, s=1/256,
  sigma2=0.1): 1e-4 for the fused form.  The composed form (per-op adjoints
  chained by autograd, alpha from a plain FP32 solve) is held to 1e-3: the
  gradient is dominated by alpha (alpha^T X), whose inner products cancel by
  about four orders of magnitude, so FP32 errors of alpha and of the Cholesky
  adjoint (measured 6e-5 and 9e-5 relative) surface at about 4e-4.
"""
import numpy as np
import pytest
import torch

from conftest import VARIANTS

pytestmark = pytest.mark.gpu

TU = lambda tr, ul: ("NT"[tr], "LU"[ul])  # noqa: E731


@pytest.fixture(scope="module")
def ag(curfp):
    import curfp_b200.autograd as ag
    return ag


def rfp_to_lower(curfp, C, tr, ul):
    """Logical lower triangle (FP64 CPU) of an RFP tensor."""
    n = curfp._n_from_rfp(C.numel())
    T = curfp.stfttr(C.detach(), transr=TU(tr, ul)[0], uplo=TU(tr, ul)[1]).double().cpu()
    return torch.tril(T.T if ul == 1 else T)


def lower_to_rfp(curfp, Lm, tr, ul):
    """RFP float32 CUDA tensor of the logical lower triangle Lm."""
    dense = (Lm.T if ul == 1 else Lm).contiguous().float().cuda()
    return curfp.strttf(dense, transr=TU(tr, ul)[0], uplo=TU(tr, ul)[1])


def spd(g, n, k=None):
    k = k or max(2, n // 2)
    X = torch.randn(n, k, generator=g, dtype=torch.float64) / k ** 0.5
    return X @ X.T + torch.eye(n, dtype=torch.float64)


# ---------------------------------------------------------------------------
# Per-op adjoints
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n", [1, 2, 5, 64, 65, 300, 700])
@pytest.mark.parametrize("tr,ul", VARIANTS)
@pytest.mark.parametrize("math", ["fp32", "bf16x3"])
def test_cholesky_adjoint_vs_dense_torch(curfp, ag, n, tr, ul, math):
    """Against torch.linalg.cholesky autograd in FP64 on the unpacked matrix:
    the symmetric input is built from its stored lower triangle P, so the
    gradient w.r.t. P is the cotangent of the stored elements."""
    if math == "bf16x3" and n < 300:
        pytest.skip("tensor-core path only engages at larger n")
    g = torch.Generator().manual_seed(31 * n + 4 * tr + ul)
    A = spd(g, n).float().double()
    W = torch.tril(torch.randn(n, n, generator=g, dtype=torch.float64)).float().double()
    P = torch.tril(A).clone().requires_grad_(True)
    L64 = torch.linalg.cholesky(torch.tril(P) + torch.tril(P, -1).T)
    (L64 * W).sum().backward()
    Ge = torch.tril(P.grad)

    C = lower_to_rfp(curfp, A, tr, ul).requires_grad_(True)
    L = ag.cholesky(C, transr=TU(tr, ul)[0], uplo=TU(tr, ul)[1], math=math)
    Wr = lower_to_rfp(curfp, W, tr, ul)
    (L * Wr).sum().backward()
    Gc = rfp_to_lower(curfp, C.grad, tr, ul)
    assert torch.linalg.norm(Gc - Ge) <= 2e-5 * torch.linalg.norm(Ge)


@pytest.mark.parametrize("n,k", [(1, 1), (17, 5), (130, 33), (600, 64)])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_ssfrk_adjoint(curfp, ag, n, k, tr, ul):
    g = torch.Generator().manual_seed(7 * n + k + 2 * tr + ul)
    A64 = torch.randn(n, k, generator=g, dtype=torch.float64).float().double()
    W = torch.tril(torch.randn(n, n, generator=g, dtype=torch.float64)).float().double()
    alpha = 0.375
    # dense FP64 reference: C = alpha A A^T, loss = <W, tril(C)>
    Ad = A64.clone().requires_grad_(True)
    ad = torch.tensor(alpha, dtype=torch.float64, requires_grad=True)
    (torch.tril(ad * Ad @ Ad.T) * W).sum().backward()

    A = A64.float().cuda().requires_grad_(True)
    at = torch.tensor(alpha, device="cuda", requires_grad=True)
    C = ag.ssfrk(A, at, transr=TU(tr, ul)[0], uplo=TU(tr, ul)[1])
    (C * lower_to_rfp(curfp, W, tr, ul)).sum().backward()
    ga = A.grad.double().cpu()
    assert torch.linalg.norm(ga - Ad.grad) <= 2e-5 * torch.linalg.norm(Ad.grad)
    assert abs(at.grad.item() - ad.grad.item()) <= 2e-5 * abs(ad.grad.item()) + 1e-6


@pytest.mark.parametrize("n,m", [(1, 1), (17, 3), (130, 1), (600, 8)])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_solve_adjoint(curfp, ag, n, m, tr, ul):
    g = torch.Generator().manual_seed(3 * n + m + 2 * tr + ul)
    L64 = torch.linalg.cholesky(spd(g, n)).float().double()
    B64 = torch.randn(n, m, generator=g, dtype=torch.float64).float().double()
    W = torch.randn(n, m, generator=g, dtype=torch.float64)
    Ld = L64.clone().requires_grad_(True)
    Bd = B64.clone().requires_grad_(True)
    X64 = torch.cholesky_solve(Bd, torch.tril(Ld))
    (X64 * W).sum().backward()

    L = lower_to_rfp(curfp, L64, tr, ul).requires_grad_(True)
    B = B64.float().cuda().requires_grad_(True)
    X = ag.solve(L, B, transr=TU(tr, ul)[0], uplo=TU(tr, ul)[1])
    (X * W.float().cuda()).sum().backward()
    gl = rfp_to_lower(curfp, L.grad, tr, ul)
    ge = torch.tril(Ld.grad)
    assert torch.linalg.norm(gl - ge) <= 2e-5 * torch.linalg.norm(ge)
    gb = B.grad.double().cpu()
    assert torch.linalg.norm(gb - Bd.grad) <= 2e-5 * torch.linalg.norm(Bd.grad)


def test_solve_vector_rhs(curfp, ag):
    n = 50
    g = torch.Generator().manual_seed(5)
    L64 = torch.linalg.cholesky(spd(g, n))
    L = lower_to_rfp(curfp, L64, 1, 1)
    y = torch.randn(n, generator=g).cuda().requires_grad_(True)
    y0 = y.detach().clone()
    x = ag.solve(L, y)
    assert x.shape == (n,)
    assert torch.equal(y.detach(), y0)  # the right-hand side is not overwritten
    ones = torch.ones(n, device="cuda")
    x.backward(ones)
    assert torch.equal(ones, torch.ones(n, device="cuda"))  # nor the incoming gradient
    ref = torch.cholesky_solve(torch.ones(n, 1, dtype=torch.float64), L64)[:, 0]
    xe = torch.cholesky_solve(y0.double().cpu()[:, None], L64)[:, 0]
    assert torch.allclose(x.detach().double().cpu(), xe, rtol=1e-5, atol=1e-6)
    assert torch.allclose(y.grad.double().cpu(), ref, rtol=1e-5, atol=1e-6)


def test_cholesky_not_pd_raises(curfp, ag):
    n = 8
    C = lower_to_rfp(curfp, -torch.eye(n, dtype=torch.float64), 1, 1)
    with pytest.raises(torch.linalg.LinAlgError):
        ag.cholesky(C)


# ---------------------------------------------------------------------------
# NLL: 1/2 y^T C^-1 y + sum log diag(L), C = s X X^T + sigma2 I
# ---------------------------------------------------------------------------
def nll64(X, s, sig2, y):
    n = X.shape[0]
    C = s * X @ X.T + sig2 * torch.eye(n, dtype=X.dtype, device=X.device)
    L = torch.linalg.cholesky(C)
    a = torch.cholesky_solve(y[:, None], L)[:, 0]
    return 0.5 * torch.dot(y, a) + torch.log(torch.diagonal(L)).sum()


def ours(ag, X, s, sig2, y, tr, ul, math, fused=True):
    Xt = X.float().cuda().requires_grad_(True)
    st = torch.tensor(s, device="cuda", requires_grad=True)
    vt = torch.tensor(sig2, device="cuda", requires_grad=True)
    loss = ag.nll(Xt, st, vt, y.float().cuda(), transr=TU(tr, ul)[0], uplo=TU(tr, ul)[1],
                  math=math, fused=fused)
    loss.backward()
    return loss.item(), Xt.grad.double().cpu(), st.grad.item(), vt.grad.item()


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("tr,ul", VARIANTS)
def test_nll_grad_vs_fd64(ag, tr, ul, fused):
    """n=256, k=32: directional FP64 central differences of the dense NLL."""
    n, k, s, sig2 = 256, 32, 1.0 / 32, 0.1
    g = torch.Generator().manual_seed(2024 + 2 * tr + ul)
    X = torch.randn(n, k, generator=g, dtype=torch.float64).float().double()
    y = torch.randn(n, generator=g, dtype=torch.float64).float().double()
    f0, gX, gs, gv = ours(ag, X, s, sig2, y, tr, ul, "fp32", fused)
    assert abs(f0 - nll64(X, s, sig2, y).item()) <= 1e-5 * abs(f0)
    h = 1e-5
    for i in range(3):
        E = torch.randn(n, k, generator=g, dtype=torch.float64)
        fd = (nll64(X + h * E, s, sig2, y) - nll64(X - h * E, s, sig2, y)).item() / (2 * h)
        an = torch.sum(gX * E).item()
        assert abs(an - fd) <= 1e-4 * torch.linalg.norm(gX).item() * torch.linalg.norm(E).item()
    fds = (nll64(X, s + h, sig2, y) - nll64(X, s - h, sig2, y)).item() / (2 * h)
    fdv = (nll64(X, s, sig2 + h, y) - nll64(X, s, sig2 - h, y)).item() / (2 * h)
    assert abs(gs - fds) <= 1e-4 * abs(fds)
    assert abs(gv - fdv) <= 1e-4 * abs(fdv)


@pytest.mark.parametrize("math,fused,tol", [("fp32", True, 1e-4), ("bf16x3", True, 1e-4),
                                            ("fp32", False, 1e-3), ("bf16x3", False, 1e-3)])
def test_nll_grad_vs_dense_torch_8192(ag, math, fused, tol):
    """The documented workload: X (8192, 256), s = 1/256, sigma2 = 0.1; the
    gradient to X, s, sigma2 against dense FP64 autograd."""
    n, d, s, sig2 = 8192, 256, 1.0 / 256, 0.1
    g = torch.Generator().manual_seed(8192)
    X = torch.randn(n, d, generator=g).double()
    y = torch.randn(n, generator=g).double()
    f, gX, gs, gv = ours(ag, X, s, sig2, y, 1, 1, math, fused)

    Xd = X.cuda().requires_grad_(True)
    sd = torch.tensor(s, dtype=torch.float64, device="cuda", requires_grad=True)
    vd = torch.tensor(sig2, dtype=torch.float64, device="cuda", requires_grad=True)
    fd = nll64(Xd, sd, vd, y.cuda())
    fd.backward()
    assert abs(f - fd.item()) <= 1e-4 * abs(fd.item())
    gXd = Xd.grad.cpu()
    rel = (torch.linalg.norm(gX - gXd) / torch.linalg.norm(gXd)).item()
    assert rel <= tol, rel
    assert abs(gs - sd.grad.item()) <= tol * abs(sd.grad.item())
    assert abs(gv - vd.grad.item()) <= tol * abs(vd.grad.item())
