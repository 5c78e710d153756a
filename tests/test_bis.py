"""Refinement solves by inverted diagonal super-blocks (ddlak_bis_*): the
persistent queue-ordered solve of L L^T X = B against numpy, in FP64 and FP32
arithmetic, for orders around the 1024-row super-block and the 64-row tile and
for 1..16 right-hand sides (two passes beyond 8)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _C():
    from libddla_b200 import ddla
    return ddla._c_api


def _k(name, restype, *argtypes):
    f = getattr(_C().lib, name)
    f.restype = restype
    f.argtypes = list(argtypes)
    return f


def _factor(n, rng):
    """FP32 lower Cholesky factor of a well-conditioned SPD matrix (column-major, ld % 4 == 0)."""
    G = rng.standard_normal((n, n))
    A = G @ G.T / n + np.eye(n)
    L = np.linalg.cholesky(A).astype(np.float32)
    ldl = (n + 3) // 4 * 4
    Lp = np.full((ldl, n), np.nan, dtype=np.float32, order="F")  # padding rows poisoned: never read
    Lp[:n, :n] = np.tril(L) + np.triu(np.full((n, n), np.nan, dtype=np.float32), 1)
    return L.astype(np.float64), Lp, ldl


@pytest.mark.parametrize("n,nrhs", [(1, 1), (5, 3), (64, 8), (1000, 8), (1024, 2), (1025, 8), (2048, 9),
                                    (3000, 16), (4100, 8), (2111, 1)])
@pytest.mark.parametrize("single", [False, True])
def test_bis_solve_matches_numpy(handle, n, nrhs, single):
    rng = np.random.default_rng(1000 * n + nrhs)
    L, Lp, ldl = _factor(n, rng)
    B = np.asfortranarray(rng.standard_normal((n, nrhs)))
    vp, i, ll, ull = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_ulonglong
    inv_bytes = _k("ddlak_bis_inverse_bytes", ull, i)(n)
    ws = _k("ddlak_bis_solve_workspace", ull, i, i)(n, nrhs)
    inverse = _k("ddlak_bis_inverse", i, i, vp, ll, vp, vp, vp)
    narrow = _k("ddlak_bis_inverse_narrow", i, i, vp, vp, vp)
    solve = _k("ddlak_bis_solve_f32" if single else "ddlak_bis_solve", i, i, i, vp, ll, vp, vp, ll, vp, ull, vp)
    st = ctypes.c_void_p()
    _C().check_status(_C().ddla_c_get_stream(handle.ptr, ctypes.byref(st)), "stream")
    ptrs = []
    try:
        dL = handle.malloc(Lp.nbytes)
        ptrs.append(dL)
        handle.memcpy(dL, Lp.ctypes.data, Lp.nbytes)
        dD = handle.malloc(inv_bytes)
        dT = handle.malloc(inv_bytes)
        dD32 = handle.malloc(inv_bytes // 2)
        dW = handle.malloc(ws)
        dB = handle.malloc(B.nbytes)
        ptrs += [dD, dT, dD32, dW, dB]
        handle.memcpy(dB, B.ctypes.data, B.nbytes)
        assert inverse(n, dL, ldl, dD, dT, st) == 0
        assert narrow(n, dD, dD32, st) == 0
        assert solve(n, nrhs, dL, ldl, dD32 if single else dD, dB, n, dW, ws, st) == 0
        X = np.empty_like(B)
        handle.memcpy(X.ctypes.data, dB, X.nbytes)
        handle.synchronize()
    finally:
        for p in ptrs:
            handle.free(p)
    Xref = np.linalg.solve(L @ L.T, B)
    rel = np.max(np.abs(X - Xref)) / np.max(np.abs(Xref))
    # FP32 arithmetic: a few units of single rounding times the order's growth; FP64: double rounding
    assert rel < (1e-4 if single else 1e-11), rel


def test_bis_solve_argument_errors(handle):
    vp, i, ll, ull = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_ulonglong
    solve = _k("ddlak_bis_solve_f32", i, i, i, vp, ll, vp, vp, ll, vp, ull, vp)
    # 17 right-hand sides, a leading dimension not a multiple of 4, too little scratch
    assert solve(100, 17, 256, 100, 256, 256, 100, 256, 1 << 30, None) != 0
    assert solve(100, 8, 256, 102, 256, 256, 100, 256, 1 << 30, None) != 0
    assert solve(100, 8, 256, 100, 256, 256, 100, 256, 16, None) != 0
    assert solve(0, 8, None, 0, None, None, 0, None, 0, None) == 0


@pytest.mark.parametrize("n,nrhs", [(1, 1), (63, 3), (1000, 8), (1024, 16), (1025, 8), (2111, 1), (3000, 9),
                                    (4100, 8)])
def test_bis_solve_fp64_factor_matches_numpy(handle, n, nrhs):
    """The same persistent solve with an FP64 factor (the plain ppotrs at large orders): the
    inverse blocks read in place from L (ddlak_bis_inverse_f64), FP64 boxes of 128 columns
    for the row units and 128 rows for the column units; the upper triangle of L's storage
    and its padding rows are NaN (never read)."""
    rng = np.random.default_rng(77 * n + nrhs)
    G = rng.standard_normal((n, n))
    L = np.linalg.cholesky(G @ G.T / n + np.eye(n))
    ldl = n + (n & 1) + 2  # even, with padding rows
    Lp = np.full((ldl, n), np.nan, order="F")
    Lp[:n, :n] = np.tril(L) + np.triu(np.full((n, n), np.nan), 1)
    B = np.asfortranarray(rng.standard_normal((n, nrhs)))
    vp, i, ll, ull = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_ulonglong
    inv_bytes = _k("ddlak_bis_inverse_bytes", ull, i)(n)
    ws = _k("ddlak_bis_solve_workspace", ull, i, i)(n, nrhs)
    inverse = _k("ddlak_bis_inverse_f64", i, i, vp, ll, vp, vp)
    solve = _k("ddlak_bis_solve_f64", i, i, i, vp, ll, vp, vp, ll, vp, ull, vp)
    st = ctypes.c_void_p()
    _C().check_status(_C().ddla_c_get_stream(handle.ptr, ctypes.byref(st)), "stream")
    ptrs = []
    try:
        dL, dD, dW, dB = handle.malloc(Lp.nbytes), handle.malloc(inv_bytes), handle.malloc(ws), handle.malloc(B.nbytes)
        ptrs += [dL, dD, dW, dB]
        handle.memcpy(dL, Lp.ctypes.data, Lp.nbytes)
        handle.memcpy(dB, B.ctypes.data, B.nbytes)
        assert inverse(n, dL, ldl, dD, st) == 0
        assert solve(n, nrhs, dL, ldl, dD, dB, n, dW, ws, st) == 0
        X = np.empty_like(B)
        status = np.zeros(1, dtype=np.int32)
        handle.memcpy(X.ctypes.data, dB, X.nbytes)
        handle.memcpy(status.ctypes.data, dW, 4)
        handle.synchronize()
    finally:
        for p in ptrs:
            handle.free(p)
    assert status[0] == 0
    Xref = np.linalg.solve(L @ L.T, B)
    assert np.max(np.abs(X - Xref)) / np.max(np.abs(Xref)) < 1e-11
