"""The benchmark configurations at their full sizes, checked through the C ABI.

* SE-kernel pposv, double and complex double, n = 16384, nrhs = 64:
  A = K + 1e-2 I with K a squared-exponential kernel (lengthscale 0.2) on points
  uniform in [0,1]^3 (complex: K exp(i k.(x - y))).  The factor's scaled backward
  error ||A - L L^H||_F / (n eps ||A||_F) <= 10 and the solution against the
  reference's CPU arm (LAPACK ?potrf + two ?trsm, oracle/lapack_arm.py).
* Mixed-precision pposv, n = 32768, nrhs = 8, A = U diag(s) U^T at kappa 1e2, 1e6,
  1e10 for both tensor-core precisions: the low-precision factor carries the solve
  (no FP64 fallback) wherever it can (kappa 1e2 and 1e6), normwise backward error
  <= 10 n eps and the forward error against the exact solution U diag(1/s) U^T B
  within what that backward error allows (kappa times it, with a margin of 10).
* The large GP likelihood, one n = 16384 FP32 problem: dloss/dtheta against FP64
  torch autograd, within a small multiple of the error torch's own FP32 gradient
  makes on the same points.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = float(np.finfo(np.float64).eps)


def _torch():
    import torch

    return torch


@pytest.mark.parametrize("p", ["d", "z"])
def test_se_kernel_pposv_n16384(handle, p):
    torch = _torch()
    from libddla_b200 import ddla
    from libddla_b200.workloads import se_kernel
    from oracle import lapack_arm

    dev = torch.device("cuda")
    n, nrhs, cplx = 16384, 64, p == "z"
    A = se_kernel(n, 0xDD1A0002, complex_=cplx, device=dev)  # Hermitian
    Acm = A.T.contiguous()  # column-major storage of A
    g = torch.Generator(device=dev).manual_seed(0xDD1A0102)
    Bt = torch.randn(nrhs, n, generator=g, device=dev, dtype=torch.float64)
    if cplx:
        Bt = torch.complex(Bt, torch.randn(nrhs, n, generator=g, device=dev, dtype=torch.float64))
    Xt = Bt.clone()
    npdt = np.complex128 if cplx else np.float64
    dA = ddla.DistributedMatrix.wrap(handle, Acm.data_ptr(), n, n, n, npdt, mb=256, nb=256)
    dX = ddla.DistributedMatrix.wrap(handle, Xt.data_ptr(), n, nrhs, n, npdt, mb=256, nb=256)
    _, info = ddla.pposv(dA, dX, "L")
    assert info == 0
    L = torch.tril(Acm.T)
    R = L @ L.conj().T
    R -= A
    bwd = float(torch.linalg.norm(R) / (n * EPS * torch.linalg.norm(A)))
    del R, L, Acm
    assert bwd <= 10, bwd
    Ah = np.asfortranarray(A.cpu().numpy())
    del A
    _, Xref, cinfo = lapack_arm.pposv(Ah, np.asfortranarray(Bt.T.cpu().numpy()), "L", overwrite=True)
    assert cinfo == 0
    X = Xt.T.cpu().numpy()
    rel = float(np.max(np.abs(X - Xref)) / np.max(np.abs(Xref)))
    print(f"se-kernel {p}: factor backward error {bwd:.3g}, solution vs LAPACK {rel:.3g}")
    assert rel <= 1e-10, rel


@pytest.fixture(scope="module")
def householder_cases():
    torch = _torch()
    from libddla_b200.workloads import householder_factors, householder_solve, householder_spd

    n, nrhs = 32768, 8
    dev = torch.device("cuda")
    g = torch.Generator(device=dev).manual_seed(0xDD1A0103)
    Bt = torch.randn(nrhs, n, generator=g, device=dev, dtype=torch.float64)
    cache = {}

    def get(kappa):
        if kappa not in cache:
            cache.clear()
            torch.cuda.empty_cache()
            A = householder_spd(n, kappa, 0xDD1A0003, device=dev)
            s, vs = householder_factors(n, kappa, 0xDD1A0003, device=dev)
            cache[kappa] = (A, householder_solve(s, vs, Bt.T))
        return cache[kappa]

    yield n, nrhs, Bt, get
    cache.clear()
    torch.cuda.empty_cache()


# (precision, kappa) pairs whose low-precision factor must carry the solve (no FP64 fallback).
# At kappa = 1e10 both factors need a diagonal shift (2^-10 relative for TF32, 2^-7 for BF16)
# far above 1/kappa, so GMRES-IR does not reach FP64 accuracy in 30 sweeps and the routine
# takes its FP64 fallback (LAPACK ?sposv's behaviour); the answer must be as accurate anyway.
MIXED_CONVERGES = {("T", 1e2), ("T", 1e6), ("B", 1e2), ("B", 1e6)}


@pytest.mark.parametrize("kappa", [1e2, 1e6, 1e10])
@pytest.mark.parametrize("prec", ["T", "B"])
def test_mixed_pposv_n32768(handle, householder_cases, prec, kappa):
    torch = _torch()
    from libddla_b200 import ddla

    n, nrhs, Bt, get = householder_cases
    A, Xex = get(kappa)
    Acopy = A.clone()
    Xt = torch.empty_like(Bt)
    wrap = lambda t, rows, cols: ddla.DistributedMatrix.wrap(handle, t.data_ptr(), rows, cols, n, np.float64,
                                                            mb=256, nb=256)
    dA, dB, dX = wrap(Acopy, n, n), wrap(Bt, n, nrhs), wrap(Xt, n, nrhs)
    _, info, rep = ddla.pposv_mixed(dA, dB, dX, precision=prec)
    assert info == 0
    X = Xt.T
    an = float(A.abs().sum(dim=0).max())
    R = Bt.T - A @ X
    bwd = float((R.abs().max(dim=0).values / (an * X.abs().max(dim=0).values)).max())
    fwd = float(((X - Xex).abs().max(dim=0).values / Xex.abs().max(dim=0).values).max())
    print(f"mixed {prec} kappa={kappa:g}: {rep} backward {bwd:.3g} forward {fwd:.3g}")
    if (prec, kappa) in MIXED_CONVERGES:
        assert rep["iter"] >= 0, rep  # the tensor-core factor carried the solve
        assert bool(torch.equal(Acopy, A))  # A left unchanged
    assert bwd <= 10 * n * EPS, (bwd, rep)
    # forward error of a solution with normwise backward error bwd: at most about kappa * bwd
    assert fwd <= 10 * kappa * max(bwd, EPS), (fwd, bwd, rep)


def test_gp_large_f32_gradient(handle):
    torch = _torch()
    from libddla_b200.ddla import autograd as ag

    dev = torch.device("cuda")
    n = 16384
    g = torch.Generator(device=dev).manual_seed(0xDD1A0005)
    X = torch.rand(1, n, 2, generator=g, device=dev, dtype=torch.float32)
    y = torch.randn(1, n, generator=g, device=dev, dtype=torch.float32)
    th = torch.tensor([0.3, 1.0, 1e-2], dtype=torch.float64, device=dev, requires_grad=True)
    loss = ag.gp_nll(X, y, th).sum()
    loss.backward()
    ours = th.grad.detach().clone()

    def torch_grad(dt):
        t = torch.tensor([0.3, 1.0, 1e-2], dtype=torch.float64, device=dev, requires_grad=True)
        Xd = X[0].to(dt)
        K = t[1].to(dt) * torch.exp(-torch.cdist(Xd, Xd).square_() / (2 * t[0].to(dt) ** 2))
        K = K + t[2].to(dt) * torch.eye(n, dtype=dt, device=dev)
        L = torch.linalg.cholesky(K)
        del K
        yd = y[0].to(dt)
        a = torch.cholesky_solve(yd.unsqueeze(-1), L).squeeze(-1)
        lo = 0.5 * ((yd * a).sum() + 2 * torch.log(torch.diagonal(L)).sum())
        lo.backward()
        return float(lo), t.grad.detach().clone()

    l64, g64 = torch_grad(torch.float64)
    torch.cuda.empty_cache()
    _, g32 = torch_grad(torch.float32)
    torch.cuda.empty_cache()
    err = float(((ours - g64).abs() / g64.abs()).max())
    err32 = float(((g32 - g64).abs() / g64.abs()).max())
    print(f"gp n=16384 f32: grad rel err vs fp64 {err:.3g} (torch fp32 {err32:.3g}); loss {float(loss):.6g} vs {l64:.6g}")
    assert abs(float(loss) - l64) <= 1e-3 * abs(l64)
    assert err <= max(4 * err32, 1e-4), (err, err32)
