"""Mixed-precision path: tensor-core factorization, FP64 residual kernel and pposv_mixed (GPU)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ddla():
    from libddla_b200 import ddla

    return ddla


def _spd(rng, n, shift=1.0):
    G = rng.standard_normal((n, n))
    return G @ G.T / n + shift * np.eye(n)


def _dev(handle, arr_f, nbytes=None):
    """Device copy of a Fortran-ordered host array; returns the pointer."""
    p = handle.malloc(nbytes or arr_f.nbytes)
    handle.memcpy(p, arr_f.ctypes.data, arr_f.nbytes)
    handle.synchronize()
    return p


def _stream(handle):
    C = _ddla()._c_api
    s = ctypes.c_void_p()
    C.check_status(C.ddla_c_get_stream(handle.ptr, ctypes.byref(s)), "stream")
    return s


def _k(name, *argtypes):
    C = _ddla()._c_api
    f = getattr(C.lib, name)
    f.restype = ctypes.c_int
    f.argtypes = list(argtypes)
    return f


@pytest.mark.parametrize("n,nrhs,pad", [(200, 3, 0), (777, 20, 0), (1030, 8, 0), (1, 1, 1), (64, 8, 0), (67, 1, 1),
                                        (68, 7, 2), (131, 8, 5), (2049, 5, 1), (4100, 8, 12), (333, 16, 1),
                                        (500, 9, 0)])
def test_symm_residual_matches_numpy(handle, n, nrhs, pad):
    """Every residual kernel: DMMA (nrhs <= 8, even leading dimensions), TMA
    (nrhs <= 16), element copies (odd leading dimensions); ragged last tiles."""
    rng = np.random.default_rng(n)
    A = _spd(rng, n)
    ld = n + pad
    Al = np.full((ld, n), np.nan, order="F")  # upper triangle and padding poisoned: never read
    Al[:n, :n] = np.tril(A) + np.triu(np.full((n, n), np.nan), 1)
    X = np.asfortranarray(rng.standard_normal((n, nrhs)))
    B = np.asfortranarray(rng.standard_normal((n, nrhs)))
    vp, i, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
    f = _k("ddlak_symm_residual", i, i, vp, ll, vp, ll, vp, ll, vp, ll, vp)
    dA, dX, dB = _dev(handle, Al), _dev(handle, X), _dev(handle, B)
    dR = handle.malloc(B.nbytes)
    try:
        assert f(n, nrhs, dA, ld, dX, n, dB, n, dR, n, _stream(handle)) == 0
        R = np.empty_like(B)
        handle.memcpy(R.ctypes.data, dR, R.nbytes)
        handle.synchronize()
        ref = B - A @ X
        assert np.all(np.isfinite(R))
        assert np.max(np.abs(R - ref)) <= 1e-12 * np.max(np.abs(A)) * np.max(np.abs(X)) * n
    finally:
        for p in (dA, dX, dB, dR):
            handle.free(p)


@pytest.mark.parametrize("precision,tol", [("B", 3e-2), ("T", 4e-3)])
@pytest.mark.parametrize("n", [128, 300, 1111, 2048, 4700, 5000])
def test_tensor_core_factorization(handle, precision, tol, n):
    """ddlak_potrf_mixed: backward error of the FP32 factor at the level of the operand rounding
    (n=4700 and 5000: their first trailing updates run on CTA pairs, 256 x 256 blocks; at 4700
    the first one covers 33 tile rows, so the last pair's second CTA holds rows past the end)."""
    rng = np.random.default_rng(7 + n)
    A = _spd(rng, n)
    ldw = (n + 3) // 4 * 4
    W = np.zeros((ldw, n), dtype=np.float32, order="F")
    W[:n, :n] = np.tril(A).astype(np.float32)
    vp, i, ll, c = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_char
    pb = _k("ddlak_mixed_panel_bytes", i)
    pb.restype = ctypes.c_ulonglong
    f = _k("ddlak_potrf_mixed", c, i, vp, ll, vp, vp, vp, vp, vp)
    dW = _dev(handle, W)
    P0, P1 = handle.malloc(pb(n)), handle.malloc(pb(n))
    dI = handle.malloc(256)
    try:
        assert f(precision.encode(), n, dW, ldw, P0, P1, dI, dI + 4, _stream(handle)) == 0
        out = np.zeros(2, dtype=np.int32)
        handle.memcpy(out.ctypes.data, dI, 8)
        handle.memcpy(W.ctypes.data, dW, W.nbytes)
        handle.synchronize()
        assert out[1] == 0, "tensor-core pipeline wait gave up"
        assert out[0] == 0
        L = np.tril(W[:n, :n]).astype(np.float64)
        err = np.linalg.norm(A - L @ L.T) / np.linalg.norm(A)
        assert err < tol, err
        Lref = np.linalg.cholesky(A)
        assert np.max(np.abs(L - Lref)) / np.max(np.abs(Lref)) < 10 * tol
    finally:
        for p in (dW, P0, P1, dI):
            handle.free(p)


@pytest.mark.parametrize("precision", ["B", "T"])
def test_tensor_core_factorization_failed_pivot_on_cta_pairs(handle, precision):
    """A failed pivot in the first block column at n=4700: the trailing updates that follow
    run on CTA pairs, which take no early exit, over the failed factor; the order of the
    failed minor comes back and no pipeline wait gives up."""
    n = 4700
    ldw = (n + 3) // 4 * 4
    W = np.zeros((ldw, n), dtype=np.float32, order="F")
    W[np.arange(n), np.arange(n)] = 2.0
    W[100, 100] = -1.0
    vp, i, ll, c = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_char
    pb = _k("ddlak_mixed_panel_bytes", i)
    pb.restype = ctypes.c_ulonglong
    f = _k("ddlak_potrf_mixed", c, i, vp, ll, vp, vp, vp, vp, vp)
    dW = _dev(handle, W)
    P0, P1 = handle.malloc(pb(n)), handle.malloc(pb(n))
    dI = handle.malloc(256)
    try:
        assert f(precision.encode(), n, dW, ldw, P0, P1, dI, dI + 4, _stream(handle)) == 0
        out = np.zeros(2, dtype=np.int32)
        handle.memcpy(out.ctypes.data, dI, 8)
        handle.synchronize()
        assert out[1] == 0, "tensor-core pipeline wait gave up"
        assert out[0] == 101
    finally:
        for p in (dW, P0, P1, dI):
            handle.free(p)


def _householder_spd(n, kappa, seed):
    from libddla_b200.workloads import householder_spd_host

    return householder_spd_host(n, kappa, seed)


def _householder_exact_solve(n, kappa, seed, B):
    """x* = A^-1 B for A = householder_spd_host(n, kappa, seed) = H1 H2 H3 H4 diag(s) H4 H3 H2 H1:
    the same reflectors and spectrum, applied to B (orthogonal steps and one diagonal scaling,
    so x* carries only a few units of rounding)."""
    rng = np.random.default_rng(seed)
    s = float(kappa) ** (-np.arange(n) / max(1, n - 1))
    vs = [rng.standard_normal(n) for _ in range(4)]

    def refl(v, Z):
        return Z - (2.0 / (v @ v)) * np.outer(v, v @ Z)

    Z = np.array(B, dtype=np.float64)
    for v in vs:  # H4 H3 H2 H1 B
        Z = refl(v, Z)
    Z = Z / s[:, None]
    for v in reversed(vs):  # H1 H2 H3 H4 (.)
        Z = refl(v, Z)
    return Z


@pytest.mark.parametrize("precision", ["B", "T"])
@pytest.mark.parametrize("kappa", [1e2, 1e6, 1e10])
def test_pposv_mixed_reaches_fp64_accuracy(handle, precision, kappa):
    """Backward error at the ?sposv stopping test, forward error against the exact solution
    within 10 kappa sqrt(n) eps (5e-12 at kappa = 1e2, 5e-8 at 1e6, 5e-4 at 1e10: an
    unrefined low-precision solution misses it by orders of magnitude), and where the
    operand precision allows it the solution must come from the refinement, not the FP64
    fallback (rep["iter"] >= 0): TF32 up to kappa = 1e6, BF16 at 1e2."""
    ddla = _ddla()
    n, nrhs = 2048, 8
    A = _householder_spd(n, kappa, 123)
    rng = np.random.default_rng(5)
    B = rng.standard_normal((n, nrhs))
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=256, nb=256)
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=256, nb=256)
    dX = ddla.DistributedMatrix(handle, n, nrhs, mb=256, nb=256)
    X, info, rep = ddla.pposv_mixed(dA, dB, dX, precision=precision)
    assert info == 0
    Xh = X.to_global_matrix()
    eps = np.finfo(np.float64).eps / 2
    anrm = np.max(np.sum(np.abs(A), axis=0))
    R = B - A @ Xh
    bwd = np.max(np.max(np.abs(R), axis=0) / (anrm * np.max(np.abs(Xh), axis=0)))
    # the ?sposv stopping test (or the FP64 fallback, whose solution meets a similar bound)
    assert bwd <= 10 * n * eps, (bwd, rep)
    # converged in mixed precision, no FP64 fallback: TF32 (u = 2^-11) up to kappa = 1e6,
    # BF16 (u = 2^-8, kappa u = 4e3 at 1e6, where GMRES-IR may or may not rescue it at this
    # order) at kappa = 1e2
    if kappa <= (1e6 if precision == "T" else 1e2):
        assert rep["iter"] >= 0, rep
    if rep["iter"] >= 0:
        np.testing.assert_array_equal(np.tril(dA.to_global_matrix()), np.tril(A))  # A unchanged
    Xexact = _householder_exact_solve(n, kappa, 123, B)
    rel = np.max(np.abs(Xh - Xexact)) / np.max(np.abs(Xexact))
    # forward error <= kappa x backward error, the latter at most ~sqrt(n) eps after the
    # ?sposv stopping test: an unrefined TF32/BF16 solution (kappa x 5e-4) is far outside
    assert rel <= 10 * kappa * np.sqrt(n) * eps + 1e-14, (rel, rep)


def test_pposv_mixed_fp64_precision_matches_pposv(handle):
    ddla = _ddla()
    n, nrhs = 700, 4
    rng = np.random.default_rng(9)
    A = _spd(rng, n)
    B = rng.standard_normal((n, nrhs))
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=64, nb=64)
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=64, nb=64)
    dX = ddla.DistributedMatrix(handle, n, nrhs, mb=64, nb=64)
    X, info, rep = ddla.pposv_mixed(dA, dB, dX, precision="D")
    assert info == 0 and rep["iter"] == 0
    dA2 = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=64, nb=64)
    dB2 = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=64, nb=64)
    X2, info2 = ddla.pposv(dA2, dB2, "L")
    np.testing.assert_allclose(X.to_global_matrix(), X2.to_global_matrix(), rtol=0, atol=1e-13)


def test_pposv_mixed_not_positive_definite_falls_back(handle):
    ddla = _ddla()
    n = 300
    A = np.eye(n)
    A[200, 200] = -1.0
    B = np.ones((n, 2))
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=64, nb=64)
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=64, nb=64)
    dX = ddla.DistributedMatrix(handle, n, 2, mb=64, nb=64)
    _, info, rep = ddla.pposv_mixed(dA, dB, dX, precision="B")
    assert info == 201
    assert rep["iter"] < 0


@pytest.mark.parametrize("group", [1, 3, 5, 8])
def test_grouped_tensor_core_factorization(handle, group):
    """ddlak_potrf_mixed_grouped: every super-step width up to the maximum gives a factor
    at the TF32 rounding level, on an order that fills no super-step exactly."""
    n = 1500
    rng = np.random.default_rng(40 + group)
    A = _spd(rng, n)
    ldw = (n + 3) // 4 * 4
    W = np.zeros((ldw, n), dtype=np.float32, order="F")
    W[:n, :n] = np.tril(A).astype(np.float32)
    vp, i, ll, c = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_char
    pb = _k("ddlak_mixed_panel_bytes", i)
    pb.restype = ctypes.c_ulonglong
    f = _k("ddlak_potrf_mixed_grouped", c, i, i, vp, ll, vp, vp, vp, vp, vp)
    dW = _dev(handle, W)
    P0, P1 = handle.malloc(pb(n)), handle.malloc(pb(n))
    dI = handle.malloc(256)
    try:
        assert f(b"T", group, n, dW, ldw, P0, P1, dI, dI + 4, _stream(handle)) == 0
        out = np.zeros(2, dtype=np.int32)
        handle.memcpy(out.ctypes.data, dI, 8)
        handle.memcpy(W.ctypes.data, dW, W.nbytes)
        handle.synchronize()
        assert out[1] == 0 and out[0] == 0, out
        L = np.tril(W[:n, :n]).astype(np.float64)
        assert np.linalg.norm(A - L @ L.T) / np.linalg.norm(A) < 4e-3
    finally:
        for p in (dW, P0, P1, dI):
            handle.free(p)
