"""pposv_mixed_host: the mixed-precision solve with A, B and X in host memory,
A streamed to the device by column panels while the arrived panels are
factored (left-looking, ddlak_potrf_mixed_stream).

* Solutions reach the ?sposv stopping test and FP64 accuracy against the
  oracle's solution (the restatement of the reference's CPU arm), for orders
  below, at and between the 512-column panels and both tensor-core precisions.
* Only A's lower triangle is read: the host upper triangle is NaN.
* The host routine and the device routine pposv_mixed agree to FP64 accuracy.
* A matrix that is not positive definite ends on the FP64 path with its info.
* Pinned host memory (torch pin_memory) takes the overlapped path.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps / 2


def _ddla():
    from libddla_b200 import ddla

    return ddla


def _poisoned(A):
    Ah = np.asfortranarray(np.tril(A) + np.triu(np.full(A.shape, np.nan), 1))
    return Ah


def _check(A, B, X, rep, info, kappa=1e4):
    from oracle import restated

    n = A.shape[0]
    assert info == 0, (info, rep)
    anrm = np.max(np.sum(np.abs(A), axis=0))
    R = B - A @ X
    bwd = np.max(np.max(np.abs(R), axis=0) / (anrm * np.max(np.abs(X), axis=0)))
    assert bwd <= 10 * n * EPS, (bwd, rep)
    _, Xref, rinfo = restated.pposv(A, B, "L")
    assert rinfo == 0
    rel = np.max(np.abs(X - Xref)) / np.max(np.abs(Xref))
    assert rel <= 10 * kappa * max(bwd, EPS) * n, (rel, rep)
    return rel


@pytest.mark.parametrize("precision", ["T", "B"])
@pytest.mark.parametrize("n,nrhs", [(100, 3), (512, 8), (600, 1), (1111, 8), (2100, 16), (4100, 5)])
def test_host_solve_reaches_fp64_accuracy(handle, precision, n, nrhs):
    from libddla_b200.workloads import householder_spd_host

    ddla = _ddla()
    A = householder_spd_host(n, 1e4, 31 + n)
    B = np.asfortranarray(np.random.default_rng(n).standard_normal((n, nrhs)))
    X, info, rep = ddla.pposv_mixed_host(handle, _poisoned(A), B, precision=precision)
    assert rep["iter"] >= 0, rep  # the tensor-core factor carried the solve
    _check(A, B, X, rep, info)


def test_host_and_device_routines_agree(handle):
    from libddla_b200.workloads import householder_spd_host

    ddla = _ddla()
    n, nrhs = 3000, 8
    A = householder_spd_host(n, 1e6, 5)
    B = np.asfortranarray(np.random.default_rng(1).standard_normal((n, nrhs)))
    Xh, info, rep = ddla.pposv_mixed_host(handle, _poisoned(A), B, precision="T")
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=256, nb=256)
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=256, nb=256)
    dX = ddla.DistributedMatrix(handle, n, nrhs, mb=256, nb=256)
    Xd, info_d, rep_d = ddla.pposv_mixed(dA, dB, dX, precision="T")
    assert info == info_d == 0 and rep["iter"] >= 0 and rep_d["iter"] >= 0
    Xd = Xd.to_global_matrix()
    _check(A, B, Xh, rep, info, kappa=1e6)
    assert np.max(np.abs(Xh - Xd)) <= 1e-9 * np.max(np.abs(Xd)), (rep, rep_d)


def test_host_fp64_precision_and_not_positive_definite(handle):
    ddla = _ddla()
    rng = np.random.default_rng(3)
    n = 700
    G = rng.standard_normal((n, n))
    A = G @ G.T / n + np.eye(n)
    B = np.asfortranarray(rng.standard_normal((n, 4)))
    X, info, rep = ddla.pposv_mixed_host(handle, _poisoned(A), B, precision="D")
    assert rep["iter"] == 0
    _check(A, B, X, rep, info, kappa=1e3)
    Abad = np.eye(n)
    Abad[200, 200] = -1.0
    _, info, rep = ddla.pposv_mixed_host(handle, _poisoned(Abad), np.ones((n, 2), order="F"), precision="B")
    assert info == 201 and rep["iter"] < 0


def test_host_solve_from_pinned_memory(handle):
    import torch

    from libddla_b200.workloads import householder_spd_host

    ddla = _ddla()
    n, nrhs = 5000, 8
    A = householder_spd_host(n, 1e5, 77)
    At = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
    At.copy_(torch.from_numpy(np.ascontiguousarray(A.T)))  # row-major storage of A^T = column-major A
    Bt = torch.empty((nrhs, n), dtype=torch.float64, pin_memory=True)
    B = np.random.default_rng(2).standard_normal((n, nrhs))
    Bt.copy_(torch.from_numpy(np.ascontiguousarray(B.T)))
    Xt = torch.empty((nrhs, n), dtype=torch.float64, pin_memory=True)
    X, info, rep = ddla.pposv_mixed_host(handle, At.numpy().T, Bt.numpy().T, precision="T", X=Xt.numpy().T)
    assert X.ctypes.data == Xt.data_ptr()
    _check(A, B, Xt.numpy().T, rep, info, kappa=1e5)
