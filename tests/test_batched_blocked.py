"""Batched blocked FP64 Cholesky (ddlak_potrf_batched_f64) and the batched
substitution with log-determinant (ddlak_potrs_batched_f64), the forward of the
equal-order likelihood batches from order 512: factors, solutions and log det
against numpy per matrix, block-edge orders, and a matrix that is not positive
definite inside a batch (LAPACK info, b kept, log det NaN, the other matrices
unaffected)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fns():
    from libddla_b200.ddla import _c_api as C
    f = C.lib.ddlak_potrf_batched_f64
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_void_p,
                  ctypes.c_void_p]
    s = C.lib.ddlak_potrs_batched_f64
    s.restype = ctypes.c_int
    s.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_void_p,
                  ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return f, s


def _spd(batch, n, seed):
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((batch, n, n))
    A = G @ G.transpose(0, 2, 1) / n + 0.1 * np.eye(n)
    b = rng.standard_normal((batch, n))
    return A, b


def _run(A, b, poison_upper=True):
    import torch
    batch, n, _ = A.shape
    # column-major per matrix: store A^T row-major (A is symmetric, the lower triangle is read)
    Ad = torch.tensor(np.ascontiguousarray(A.transpose(0, 2, 1)), device="cuda")
    if poison_upper:
        up = torch.triu(torch.ones(n, n, dtype=torch.bool, device="cuda"), 1)
        Ad.transpose(1, 2)[:, up] = float("nan")  # entries above the diagonal in the column-major view
    bd = torch.tensor(b, device="cuda")
    info = torch.full((batch,), -7, dtype=torch.int32, device="cuda")
    logdet = torch.zeros(batch, dtype=torch.float64, device="cuda")
    f, s = _fns()
    torch.cuda.synchronize()
    assert f(batch, n, Ad.data_ptr(), n, n * n, info.data_ptr(), None) == 0
    assert s(batch, n, Ad.data_ptr(), n, n * n, bd.data_ptr(), n, info.data_ptr(), logdet.data_ptr(), None) == 0
    torch.cuda.synchronize()
    L = Ad.transpose(1, 2).cpu().numpy()  # back to (row, col)
    return L, bd.cpu().numpy(), info.cpu().numpy(), logdet.cpu().numpy()


@pytest.mark.parametrize("n,batch", [(2, 3), (130, 2), (512, 4), (520, 3), (1000, 2), (1024, 3)])
def test_batched_blocked_matches_numpy(n, batch):
    A, b = _spd(batch, n, 9000 + n)
    L, x, info, logdet = _run(A, b)
    assert (info == 0).all()
    for m in range(batch):
        Lr = np.linalg.cholesky(A[m])
        low = np.tril(np.ones((n, n), dtype=bool))
        assert np.isfinite(L[m][low]).all()
        assert np.abs(L[m][low] - Lr[low]).max() <= 1e-12 * np.abs(Lr).max()
        xr = np.linalg.solve(A[m], b[m])
        assert np.abs(x[m] - xr).max() <= 1e-10 * np.abs(xr).max()
        ld = 2.0 * np.log(np.diag(Lr)).sum()
        assert abs(logdet[m] - ld) <= 1e-12 * max(1.0, abs(ld))


def test_batched_blocked_failure_is_per_matrix():
    n, batch = 600, 3
    A, b = _spd(batch, n, 4242)
    A[1, 300, 300] = -1.0  # leading minor of order 301 is not positive
    L, x, info, logdet = _run(A, b)
    assert info[0] == 0 and info[2] == 0
    assert info[1] == 301
    assert np.array_equal(x[1], b[1])
    assert np.isnan(logdet[1])
    for m in (0, 2):
        xr = np.linalg.solve(A[m], b[m])
        assert np.abs(x[m] - xr).max() <= 1e-10 * np.abs(xr).max()
    # columns before the failed block column are final (LAPACK's blocked dpotrf)
    Lr = np.linalg.cholesky(A[1][:256, :256])
    assert np.abs(L[1][:256, :256][np.tril_indices(256)] - Lr[np.tril_indices(256)]).max() <= 1e-12


def test_batched_blocked_rejects_odd_leading_dimension():
    import torch
    f, _ = _fns()
    n = 513
    A = torch.eye(n, dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert f(1, n, A.data_ptr(), n, n * n, info.data_ptr(), None) != 0
