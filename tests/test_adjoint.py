"""Differentiable likelihood (libddla_b200.ddla.autograd): loss and gradients of
chol_nll / gp_nll against an FP64 torch.linalg reference, central finite
differences, torch.autograd.gradcheck, the large-order path and failures."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _t():
    import torch
    return torch


def _ag():
    from libddla_b200.ddla import autograd
    return autograd


def spd(batch, n, dtype, seed):
    torch = _t()
    g = torch.Generator(device="cpu").manual_seed(seed)
    G = torch.randn(batch, n, n, generator=g, dtype=torch.float64)
    A = G @ G.transpose(1, 2) / n + 0.1 * torch.eye(n, dtype=torch.float64)
    y = torch.randn(batch, n, generator=g, dtype=torch.float64)
    return A.to(dtype).cuda(), y.to(dtype).cuda()


def ref_loss(A, y):
    """FP64 torch.linalg reference of 1/2 (y^T A^-1 y + log det A), autograd-capable."""
    torch = _t()
    A64 = A.to(torch.float64)
    y64 = y.to(torch.float64)
    alpha = torch.linalg.solve(A64, y64.unsqueeze(-1)).squeeze(-1)
    return 0.5 * ((y64 * alpha).sum(-1) + torch.linalg.slogdet(A64)[1])


def se_kernel(X, theta):
    torch = _t()
    l, sf2, s2 = theta[0], theta[1], theta[2]
    r2 = ((X[:, :, None, :] - X[:, None, :, :]) ** 2).sum(-1)
    n = X.shape[1]
    return sf2 * torch.exp(-r2 / (2 * l * l)) + s2 * torch.eye(n, dtype=X.dtype, device=X.device)


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("n", [1, 17, 64, 100, 256, 512, 1024])
def test_chol_nll_loss_and_gradient_vs_torch(n, dtype):
    torch = _t()
    dt = getattr(torch, dtype)
    batch = 3
    A, y = spd(batch, n, dt, 100 + n)
    A1 = A.clone().requires_grad_(True)
    y1 = y.clone().requires_grad_(True)
    loss = _ag().chol_nll(A1, y1)
    loss.sum().backward()
    A2 = A.to(torch.float64).clone().requires_grad_(True)
    y2 = y.to(torch.float64).clone().requires_grad_(True)
    ref = ref_loss(A2, y2)
    ref.sum().backward()
    tol = 1e-10 if dtype == "float64" else 2e-3
    assert torch.allclose(loss.double(), ref, rtol=tol, atol=tol * n), (loss, ref)
    gA, gA_ref = A1.grad.double(), A2.grad
    assert torch.allclose(gA, gA.transpose(1, 2))
    err = (gA - gA_ref).abs().max() / gA_ref.abs().max()
    assert err < (1e-9 if dtype == "float64" else 1e-2), err
    erry = (y1.grad.double() - y2.grad).abs().max() / y2.grad.abs().max()
    assert erry < (1e-10 if dtype == "float64" else 1e-3), erry


def test_chol_nll_central_differences():
    """<dloss/dA, E> against (loss(A + hE) - loss(A - hE)) / 2h for symmetric E."""
    torch = _t()
    A, y = spd(2, 200, torch.float64, 7)
    A1 = A.clone().requires_grad_(True)
    _ag().chol_nll(A1, y).sum().backward()
    g = torch.Generator(device="cpu").manual_seed(8)
    for _ in range(3):
        E = torch.randn(2, 200, 200, generator=g, dtype=torch.float64).cuda()
        E = E + E.transpose(1, 2)
        h = 1e-6
        fd = (_ag().chol_nll(A + h * E, y).sum() - _ag().chol_nll(A - h * E, y).sum()) / (2 * h)
        an = (A1.grad * E).sum()
        assert abs(float(fd - an)) <= 1e-6 * abs(float(an)) + 1e-8, (float(fd), float(an))


def test_chol_nll_gradcheck():
    torch = _t()
    A, y = spd(2, 12, torch.float64, 9)

    def f(A_, y_):
        return _ag().chol_nll(0.5 * (A_ + A_.transpose(1, 2)), y_)

    assert torch.autograd.gradcheck(f, (A.clone().requires_grad_(True), y.clone().requires_grad_(True)),
                                    eps=1e-6, atol=1e-7, rtol=1e-5)


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("shared", [True, False])
def test_gp_nll_theta_gradient(dtype, shared):
    """dloss/dtheta from the fused contraction against torch autograd through an
    FP64 kernel matrix, and against central differences in theta."""
    torch = _t()
    dt = getattr(torch, dtype)
    batch, n = 4, 300
    g = torch.Generator(device="cpu").manual_seed(31)
    X = torch.rand(batch, n, 2, generator=g, dtype=torch.float64).cuda()
    y = torch.randn(batch, n, generator=g, dtype=torch.float64).cuda()
    th0 = torch.tensor([0.3, 1.0, 1e-2], dtype=torch.float64)
    th = (th0.cuda() if shared else th0.repeat(batch, 1).cuda() * (1 + 0.1 * torch.arange(batch).cuda()[:, None]))
    th1 = th.clone().requires_grad_(True)
    y1 = y.to(dt).clone().requires_grad_(True)
    loss = _ag().gp_nll(X.to(dt), y1, th1)
    loss.sum().backward()
    # reference: FP64 torch autograd through the kernel matrix
    th2 = th.clone().requires_grad_(True)
    if shared:
        K = se_kernel(X, th2)
    else:
        K = torch.stack([se_kernel(X[b:b + 1], th2[b])[0] for b in range(batch)])
    ref = ref_loss(K, y)
    ref.sum().backward()
    tol = 1e-9 if dtype == "float64" else 5e-3
    assert torch.allclose(loss.double(), ref, rtol=tol, atol=tol)
    err = (th1.grad - th2.grad).abs().max() / th2.grad.abs().max()
    assert err < (1e-8 if dtype == "float64" else 2e-2), (th1.grad, th2.grad)
    if dtype == "float64":
        # central differences in each hyperparameter
        for c in range(3):
            h = 1e-5 * float(th0[c])
            e = torch.zeros_like(th)
            if shared:
                e[c] = h
            else:
                e[:, c] = h
            fd = (_ag().gp_nll(X, y, th + e).sum() - _ag().gp_nll(X, y, th - e).sum()) / (2 * h)
            an = th1.grad[c] if shared else th1.grad[:, c].sum()
            assert abs(float(fd - an)) <= 1e-5 * abs(float(an)) + 1e-6, (c, float(fd), float(an))


def test_large_order_single_problem():
    """Orders above the batched limit: blocked factorization, A^-1 from the fused solve."""
    torch = _t()
    A, y = spd(1, 1100, torch.float64, 55)
    A1 = A.clone().requires_grad_(True)
    loss = _ag().chol_nll(A1, y)
    loss.sum().backward()
    A2 = A.clone().requires_grad_(True)
    ref = ref_loss(A2, y)
    ref.sum().backward()
    assert torch.allclose(loss, ref, rtol=1e-10, atol=1e-9)
    err = (A1.grad - A2.grad).abs().max() / A2.grad.abs().max()
    assert err < 1e-9, err
    X = torch.rand(1, 1500, 2, dtype=torch.float64).cuda()
    yg = torch.randn(1, 1500, dtype=torch.float64).cuda()
    th = torch.tensor([0.3, 1.0, 1e-2], dtype=torch.float64, device="cuda", requires_grad=True)
    _ag().gp_nll(X, yg, th).sum().backward()
    th2 = th.detach().clone().requires_grad_(True)
    ref_loss(se_kernel(X, th2), yg).sum().backward()
    assert ((th.grad - th2.grad).abs().max() / th2.grad.abs().max()) < 1e-8


@pytest.mark.parametrize("n", [50, 600])
def test_not_positive_definite_raises(n):
    torch = _t()
    A, y = spd(3, n, torch.float64, 3)
    A[1, 10, 10] = -5.0
    with pytest.raises(RuntimeError, match="matrix 1"):
        _ag().chol_nll(A, y)


@pytest.mark.parametrize("n,batch", [(1, 3), (15, 2), (17, 5), (33, 1), (64, 2), (65, 3), (100, 4), (129, 2),
                                     (255, 2), (512, 1), (640, 2), (1000, 3), (1024, 2)])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_trtri_batched_inverse(n, batch, dtype):
    """ddlak_trtri_batched (W = L^-1, the lower triangle) against the inverse
    of the same factor, at orders that do and do not fill the 16-column block columns and
    32-row blocks, with batches small enough that each matrix is split over several CTAs."""
    import ctypes

    torch = _t()
    from libddla_b200.ddla import _c_api as C

    dt = getattr(torch, dtype)
    A, _ = spd(batch, n, torch.float64, 500 + n)
    Lf = torch.linalg.cholesky(A)
    L = Lf.to(dt).transpose(1, 2).contiguous().transpose(1, 2)  # column-major per matrix
    L = L.permute(0, 2, 1).contiguous()  # row-major storage of L^T = column-major L
    W = torch.full_like(L, float("nan"))
    f = C.lib.ddlak_trtri_batched
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_char, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong,
                  ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_void_p]
    torch.cuda.synchronize()
    assert f(b"d" if dtype == "float64" else b"s", batch, n, L.data_ptr(), n, n * n, W.data_ptr(), n, n * n,
             None) == 0
    torch.cuda.synchronize()
    Wc = W.permute(0, 2, 1).double()  # back to (row, col) indexing
    ref = torch.linalg.inv(L.permute(0, 2, 1).double())
    low = torch.tril(torch.ones(n, n, dtype=torch.bool, device=W.device))
    assert bool(torch.isfinite(Wc[:, low]).all())
    err = (Wc[:, low] - ref[:, low]).abs().max() / ref.abs().max()
    assert err < (1e-12 if dtype == "float64" else 1e-4), err
