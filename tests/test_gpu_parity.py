"""Parity of the sm_100a Cholesky path with the oracle and the reference tests' known answers.

Every call goes through the C ABI (libddla_c.so) via the ddla binding; the oracle
is only the checker.
"""
import ctypes
import math

import numpy as np
import pytest

import generators as G
from oracle import lapack_arm, restated

pytestmark = pytest.mark.gpu

TOL_FACTOR = {"s": 2e-5, "c": 2e-5, "d": 3e-12, "z": 3e-12}


def _ddla():
    from libddla_b200 import ddla

    return ddla


def upload_padded(h, A, n_desc, lld_extra=0, mb=8, fill=None):
    """Device matrix whose descriptor is n_desc x n_desc with LLD_ padded by lld_extra; A sits at (0,0)."""
    ddla = _ddla()
    M = ddla.DistributedMatrix(h, n_desc, n_desc, mb=mb, nb=mb, dtype=A.dtype,
                               lld=max(1, n_desc) + lld_extra)
    host = np.empty((M.lld, max(1, n_desc)), dtype=A.dtype, order="F")
    host[...] = G._scalar(A.dtype, -731, 19) if fill is None else fill
    n = A.shape[0]
    host[:n, :n] = A
    M.from_host(host, full_lld=True)
    return M, host


# --------------------------------------------------------------------------
# test_ppotrf_grids.cpp: analytic factor, padded LLD, bit-preserved outside
# --------------------------------------------------------------------------
@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("n", [1, 2, 17, 38, 129, 257])
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_ppotrf_kat_padded(handle, golden, p, n, uplo):
    ddla = _ddla()
    dt = G.DTYPES[p]
    A = golden["kat"][f"{p}_{n}_A"] if f"{p}_{n}_A" in golden["kat"].files else G.kat_matrix(n, dt)
    L = golden["kat"][f"{p}_{n}_L"] if f"{p}_{n}_L" in golden["kat"].files else G.kat_factor(n, dt)
    poisoned = A.copy()
    iu = np.triu_indices(n, 1) if uplo == "L" else np.tril_indices(n, -1)
    poisoned[iu] = np.nan  # the opposite triangle must never be read
    # the descriptor describes (n+3) x (n+3) with LLD_ + 3; factor the leading n x n only
    M, host = upload_padded(handle, poisoned, n + 3, lld_extra=3)
    info_c = ctypes.c_int(-1)
    f = getattr(ddla._c_api.lib, f"ddla_{p}_ppotrf")
    ddla._c_api.check_status(f(handle.ptr, uplo.encode(), n, M.data_ptr, 1, 1, M.desc.ctypes.data,
                               ctypes.byref(info_c)), "ppotrf")
    assert info_c.value == 0
    out = M.to_host(full_lld=True)
    want = L if uplo == "L" else L.conj().T
    got = np.tril(out[:n, :n]) if uplo == "L" else np.triu(out[:n, :n])
    err = np.max(np.abs(got - want) / (1 + np.abs(want)))
    assert err < TOL_FACTOR[p], err
    # everything outside the leading n x n (rows n.., padding, columns n..) is bit-identical
    mask = np.ones(out.shape, dtype=bool)
    mask[:n, :n] = False
    assert np.array_equal(out[mask].view(np.uint8), host[mask].view(np.uint8))


@pytest.mark.parametrize("p", ["d", "z"])
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_ppotrf_run_exact_workspace_guards(handle, golden, p, uplo):
    """ppotrf_run on caller scratch: 256-byte 0x57 guard zones stay intact (test_ppotrf_grids.cpp:77-85)."""
    ddla = _ddla()
    C = ddla._c_api
    n = 129
    A = golden["kat"][f"{p}_{n}_A"]
    M, host = upload_padded(handle, A, n, lld_extra=0)
    nbytes = ctypes.c_longlong()
    C.check_status(getattr(C.lib, f"ddla_{p}_ppotrf_workspace_size")(handle.ptr, uplo.encode(), n,
                                                                      M.desc.ctypes.data, ctypes.byref(nbytes)), "ws")
    guard = 256
    total = nbytes.value + 2 * guard
    work = handle.malloc(total)
    try:
        handle.memset(work, 0x57, total)
        for _ in range(2):
            M.from_host(host, full_lld=True)
            info = ctypes.c_int(-1)
            C.check_status(getattr(C.lib, f"ddla_{p}_ppotrf_run")(handle.ptr, uplo.encode(), n, M.data_ptr,
                                                                   M.desc.ctypes.data, ctypes.byref(info),
                                                                   work + guard, nbytes.value), "run")
            assert info.value == 0
            edge = np.zeros(total, dtype=np.uint8)
            handle.memcpy(edge.ctypes.data, work, total)
            handle.synchronize()
            assert np.all(edge[:guard] == 0x57) and np.all(edge[guard + nbytes.value:] == 0x57)
        L = golden["kat"][f"{p}_{n}_L"]
        out = M.to_host()
        got = np.tril(out) if uplo == "L" else np.triu(out).conj().T
        assert np.max(np.abs(got - L) / (1 + np.abs(L))) < TOL_FACTOR[p]
    finally:
        handle.free(work)


# --------------------------------------------------------------------------
# solutions: test_ppotrf_real.cpp, test_api_grid_ppotrf.cpp, python tests
# --------------------------------------------------------------------------
@pytest.mark.parametrize("p", ["s", "d"])
@pytest.mark.parametrize("n", [16, 40])
def test_real_spd_ppotrf_ppotrs_and_pposv(handle, golden, p, n):
    ddla = _ddla()
    z = golden["real_spd"]
    A, X, B = z[f"{p}_{n}_A"], z[f"{p}_{n}_X"], z[f"{p}_{n}_B"]
    tol = 3e-3 if p == "s" else 1e-9
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=8, nb=8)
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=8, nb=8)
    _, info = ddla.ppotrf(dA, "L")
    assert info == 0
    ddla.ppotrs(dA, dB, "L")
    assert np.max(np.abs(dB.to_global_matrix() - X)) < tol
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=8, nb=8)
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=8, nb=8)
    _, info = ddla.pposv(dA, dB, "L")
    assert info == 0
    assert np.max(np.abs(dB.to_global_matrix() - X)) < tol


@pytest.mark.parametrize("n", [1, 24])
def test_hpd_complex(handle, golden, n):
    ddla = _ddla()
    z = golden["hpd"]
    A, X, B = z[f"z_{n}_A"], z[f"z_{n}_X"], z[f"z_{n}_B"]
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=4, nb=4)
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=4, nb=4)
    _, info = ddla.ppotrf(dA, "L")
    assert info == 0
    if n == 1:
        assert abs(dA.to_global_matrix()[0, 0] - 2.0) < 1e-12
    ddla.ppotrs(dA, dB, "L")
    assert np.max(np.abs(dB.to_global_matrix() - X)) < 5e-9


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("trans", ["N", "C"])
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_pposv_side_trans(handle, side, trans, uplo):
    """test_api_grid_pposv.cpp:16-43: trans 'C' == 'N' for Hermitian A; side 'R' solves X A = B."""
    ddla = _ddla()
    n, nrhs = 37, 3
    A = G.hpd_value(n)
    X = G.x_value(n, nrhs)
    if side == "R":
        X = X.T.copy()
        B = X @ A
    else:
        B = A @ X
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=5, nb=5)
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=5, nb=5)
    _, info = ddla.pposv(dA, dB, uplo, side=side, trans=trans)
    assert info == 0
    assert np.max(np.abs(dB.to_global_matrix() - X)) < 5e-9


def test_python_cases(handle, golden):
    ddla = _ddla()
    z = golden["python"]
    for key, tol in (("ppotrf_ppotrs", 1e-11), ("pposv", 1e-11)):
        A, X = z[f"{key}_A"], z[f"{key}_X"]
        dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=16, nb=16)
        dB = ddla.DistributedMatrix.from_global_matrix(handle, A @ X, mb=16, nb=16)
        _, info = ddla.pposv(dA, dB, "L")
        assert info == 0
        assert np.max(np.abs(dB.to_global_matrix() - X)) < tol
    for key in [k for k in z.files if k.startswith("typed_") and k.endswith("_A")]:
        _, k, ch, uplo, _ = key.split("_")
        A, X, B = z[key], z[key[:-1] + "X"], z[key[:-1] + "B"]
        dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=3, nb=3)
        dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=3, nb=3)
        _, info = ddla.ppotrf(dA, uplo)
        assert info == 0
        ddla.ppotrs(dA, dB, uplo)
        tol = 2e-4 if ch in "fF" else 1e-11
        np.testing.assert_allclose(dB.to_global_matrix(), X, atol=tol, rtol=tol)


@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("where", [8, 200])
def test_not_positive_definite(handle, p, uplo, where):
    """info = order of the first failing minor; pposv leaves B untouched (test_cholesky.py:79-92)."""
    ddla = _ddla()
    n = where + 1
    A = np.eye(n, dtype=G.DTYPES[p])
    A[-1, -1] = -1
    B = np.ones((n, 2), dtype=A.dtype)
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=3, nb=3)
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=3, nb=3)
    _, info = ddla.pposv(dA, dB, uplo)
    assert info == n
    np.testing.assert_array_equal(dB.to_global_matrix(), B)
    # a NaN pivot in the middle fails at that minor too
    A = np.eye(n, dtype=G.DTYPES[p])
    A[n // 2, n // 2] = np.nan
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=3, nb=3)
    _, info = ddla.ppotrf(dA, uplo)
    assert info == n // 2 + 1


# --------------------------------------------------------------------------
# random parity against the oracle over block-size edges
# --------------------------------------------------------------------------
def _spd(rng, n, dt, shift=1.0):
    M = rng.standard_normal((n, n))
    if np.dtype(dt).kind == "c":
        M = M + 1j * rng.standard_normal((n, n))
    return (M @ M.conj().T / n + shift * np.eye(n)).astype(dt)


def backward_error(A, F, uplo, eps):
    n = A.shape[0]
    L = np.tril(F) if uplo == "L" else np.triu(F).conj().T
    A64 = A.astype(np.complex128 if A.dtype.kind == "c" else np.float64)
    L64 = L.astype(A64.dtype)
    H = np.tril(A64) + np.tril(A64, -1).conj().T if uplo == "L" else np.triu(A64) + np.triu(A64, 1).conj().T
    return np.linalg.norm(H - L64 @ L64.conj().T) / (n * eps * np.linalg.norm(H))


@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("n", [63, 64, 65, 127, 128, 129, 255, 257, 513])
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_random_parity(handle, p, n, uplo):
    ddla = _ddla()
    rng = np.random.default_rng(1000 + n)
    dt = G.DTYPES[p]
    A = _spd(rng, n, dt)
    nrhs = 1 + n % 19
    B = rng.standard_normal((n, nrhs)).astype(dt)
    F_o, X_o, info_o = restated.pposv(A, B, uplo)
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=64, nb=64)
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=64, nb=64)
    _, info = ddla.pposv(dA, dB, uplo)
    assert info == info_o == 0
    F = dA.to_global_matrix()
    X = dB.to_global_matrix()
    eps = np.finfo(np.float32 if p in "sc" else np.float64).eps
    assert backward_error(A, F, uplo, eps) <= 10
    tri = np.tril if uplo == "L" else np.triu
    rel_f = np.max(np.abs(tri(F) - tri(F_o))) / np.max(np.abs(F_o))
    rel_x = np.max(np.abs(X - X_o)) / np.max(np.abs(X_o))
    tol = 1e-4 if p in "sc" else 1e-12
    assert rel_f < tol and rel_x < tol * 10, (rel_f, rel_x)


@pytest.mark.parametrize("nrhs", [1, 16, 17, 64, 100])
def test_solve_many_rhs(handle, nrhs):
    ddla = _ddla()
    rng = np.random.default_rng(7)
    n = 700
    A = _spd(rng, n, np.float64)
    B = rng.standard_normal((n, nrhs))
    F_o, _ = restated.potrf(A, "L")
    X_o = restated.ppotrs(F_o, B, "L")
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=32, nb=32)
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=32, nb=32)
    _, info = ddla.pposv(dA, dB, "L")
    assert info == 0
    assert np.max(np.abs(dB.to_global_matrix() - X_o)) < 1e-11 * np.max(np.abs(X_o))


def test_config1_n2048_against_lapack(handle):
    """ppotrf(L)+ppotrs, d, n=2048, nrhs=16, A = G G^T/2048 + I: backward error <= 10, solution
    within 1e-10 relative of the reference's CPU arm (LAPACK dpotrf + 2 dtrsm)."""
    ddla = _ddla()
    rng = np.random.default_rng(0xDD1A0001)
    n, nrhs = 2048, 16
    Gm = rng.standard_normal((n, n))
    A = Gm @ Gm.T / n + np.eye(n)
    B = rng.standard_normal((n, nrhs))
    F_ref, X_ref, info_ref = lapack_arm.pposv(A, B, "L")
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=256, nb=256)
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=256, nb=256)
    _, info = ddla.ppotrf(dA, "L")
    assert info == info_ref == 0
    ddla.ppotrs(dA, dB, "L")
    F = dA.to_global_matrix()
    assert backward_error(A, F, "L", np.finfo(np.float64).eps) <= 10
    X = dB.to_global_matrix()
    assert np.max(np.abs(X - X_ref)) / np.max(np.abs(X_ref)) < 1e-10


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("nrhs", [1, 8, 16])
def test_large_order_solve_against_lapack(handle, uplo, nrhs):
    """pposv d at n = 5000 (above the order where ppotrs for uplo 'L', side 'L' and up to 16
    right-hand sides switches to the persistent solve by inverted 1024-row blocks; 'U' keeps
    the fused 64-row solve): within 1e-10 relative of the reference's CPU arm, and ppotrs on
    the factor again reproduces the same solution."""
    from oracle import lapack_arm

    ddla = _ddla()
    n = 5000
    rng = np.random.default_rng(17 + nrhs)
    G = rng.standard_normal((n, n))
    A = G @ G.T / n + np.eye(n)
    B = rng.standard_normal((n, nrhs))
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=256, nb=256)
    dB = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=256, nb=256)
    _, info = ddla.pposv(dA, dB, uplo)
    assert info == 0
    X = dB.to_global_matrix()
    _, X_ref, cinfo = lapack_arm.pposv(np.asfortranarray(A), np.asfortranarray(B), uplo)
    assert cinfo == 0
    assert np.max(np.abs(X - X_ref)) / np.max(np.abs(X_ref)) < 1e-10
    dB2 = ddla.DistributedMatrix.from_global_matrix(handle, B, mb=256, nb=256)
    ddla.ppotrs(dA, dB2, uplo)
    assert np.max(np.abs(dB2.to_global_matrix() - X)) <= 1e-12 * np.max(np.abs(X))


def test_potrf_device_info(handle):
    ddla = _ddla()
    n = 300
    A = _spd(np.random.default_rng(5), n, np.float64)
    A[150, 150] = -5.0
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=32, nb=32)
    dinfo = handle.malloc(4)
    try:
        handle.memset(dinfo, 0xFF, 4)
        ddla.potrf(handle, "d", "l", n, dA.data_ptr, dA.lld, dinfo)
        info = np.zeros(1, dtype=np.int32)
        handle.memcpy(info.ctypes.data, dinfo, 4)
        handle.synchronize()
        _, info_o = restated.potrf(A, "L")
        assert info[0] == info_o
    finally:
        handle.free(dinfo)


def test_empty_and_argument_errors(handle):
    ddla = _ddla()
    C = ddla._c_api
    dA = ddla.DistributedMatrix(handle, 4, 4, mb=2, nb=2)
    info = ctypes.c_int(-1)
    assert C.ddla_d_ppotrf(handle.ptr, b"L", 0, dA.data_ptr, 1, 1, dA.desc.ctypes.data, ctypes.byref(info)) == 0
    assert info.value == 0
    for uplo, n, ia in ((b"l", 4, 1), (b"X", 4, 1), (b"L", 5, 1), (b"L", -1, 1), (b"L", 4, 2)):
        st = C.ddla_d_ppotrf(handle.ptr, uplo, n, dA.data_ptr, ia, 1, dA.desc.ctypes.data, ctypes.byref(info))
        assert st == C.STATUS_EXCEPTION
        assert "ppotrf: invalid" in C.error_string(st)
    bad = dA.desc.copy()
    bad[C.MB_] = 3
    st = C.ddla_d_ppotrf(handle.ptr, b"L", 4, dA.data_ptr, 1, 1, bad.ctypes.data, ctypes.byref(info))
    assert st == C.STATUS_EXCEPTION
    bad = dA.desc.copy()
    bad[C.LLD_] = 1
    st = C.ddla_d_ppotrf(handle.ptr, b"L", 4, dA.data_ptr, 1, 1, bad.ctypes.data, ctypes.byref(info))
    assert st == C.STATUS_EXCEPTION and "LLD_A" in C.error_string(st)
    st = C.ddla_d_ppotrs(handle.ptr, b"L", b"L", b"T", 4, 1, dA.data_ptr, dA.desc.ctypes.data, dA.data_ptr,
                         dA.desc.ctypes.data)
    assert st == C.STATUS_EXCEPTION and "ppotrs" in C.error_string(st)
    st = C.ddla_d_ppotrs(handle.ptr, b"L", b"L", b"N", 4, 0, dA.data_ptr, dA.desc.ctypes.data, dA.data_ptr,
                         dA.desc.ctypes.data)
    assert st == 0
    # a grid larger than 1x1 is not served
    h = ctypes.c_void_p()
    assert C.ddla_c_init_backend(ctypes.byref(h), C.BACKEND_GPU) == 0
    assert C.ddla_c_set(h, C.ddla_c_default_comm(), 2, 1, b"R") == C.STATUS_BACKEND_UNAVAILABLE
    C.ddla_c_destroy(ctypes.byref(h))


# --------------------------------------------------------------------------
# diag_logdet: test_diag_logdet.cpp
# --------------------------------------------------------------------------
@pytest.mark.parametrize("p", list("sdcz"))
def test_diag_logdet_cases(handle, golden, p):
    ddla = _ddla()
    C = ddla._c_api
    z = golden["logdet"]
    tol = 2e-5 if p in "sc" else 3e-12
    rdt = np.float32 if p in "sc" else np.float64
    k = 0
    while f"{p}_{k}_diag" in z.files:
        d = z[f"{p}_{k}_diag"]
        n = d.size
        lda = max(1, n) + 3
        host = np.full((lda, max(1, n)), np.nan, dtype=d.dtype, order="F")
        for i in range(n):
            host[i, i] = d[i]
        dA = ddla.DistributedMatrix(handle, lda, max(1, n), mb=4, nb=4, dtype=d.dtype, lld=lda)
        dA.from_host(host, full_lld=True)
        res = np.array([91, -13], dtype=rdt)
        st = getattr(C.lib, f"ddla_{p}_diag_logdet")(handle.ptr, n, dA.data_ptr if n else None, lda, res.ctypes.data)
        if not bool(z[f"{p}_{k}_valid"]):
            assert st == C.STATUS_EXCEPTION and "nonfinite" in C.error_string(st)
            assert res[0] == 91 and res[1] == -13
        else:
            assert st == 0
            e = z[f"{p}_{k}_expect"]
            if np.isinf(e[0]):
                assert np.isinf(res[0]) and res[0] < 0 and res[1] == 0
            else:
                assert abs(res[0] - e[0]) < tol * (1 + abs(e[0]))
                assert abs(math.remainder(float(res[1]) - e[1], 2 * math.pi)) < tol
            assert dA.to_host(full_lld=True).tobytes(order="F") == host.tobytes(order="F")
        k += 1


@pytest.mark.parametrize("p", list("sdcz"))
def test_diag_logdet_parity_and_guards(handle, p):
    ddla = _ddla()
    C = ddla._c_api
    rdt = np.float32 if p in "sc" else np.float64
    n = 1025
    A = -np.eye(n, dtype=G.DTYPES[p])
    dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=64, nb=64)
    r = ddla.diag_logdet(dA)
    assert abs(r.real) < 1e-5 and abs(r.imag - math.pi) < 1e-5
    res = np.array([91, -13], dtype=rdt)
    f = getattr(C.lib, f"ddla_{p}_diag_logdet")
    assert f(handle.ptr, -1, dA.data_ptr, n, res.ctypes.data) == C.STATUS_EXCEPTION
    assert f(handle.ptr, 2**31 - 1, dA.data_ptr, 2**31 - 1, res.ctypes.data) == C.STATUS_EXCEPTION
    assert "not representable" in C.error_string(C.STATUS_EXCEPTION)
    assert res[0] == 91 and res[1] == -13
    assert f(handle.ptr, 1, dA.data_ptr, 2**31 - 1, res.ctypes.data) == 0  # lda never addresses a later column
    assert abs(res[0]) < 1e-6 and abs(res[1] - math.pi) < 1e-6


def test_diag_logdet_random_vs_oracle(handle):
    ddla = _ddla()
    rng = np.random.default_rng(9)
    for p in "dz":
        n = 5000
        d = rng.standard_normal(n) + (1j * rng.standard_normal(n) if p == "z" else 0)
        A = np.diag(d).astype(G.DTYPES[p])
        dA = ddla.DistributedMatrix.from_global_matrix(handle, A, mb=64, nb=64)
        r = ddla.diag_logdet(dA)
        ro = restated.diag_logdet(A)
        assert abs(r.real - ro.real) < 1e-10 * abs(ro.real) + 1e-10
        assert abs(math.remainder(r.imag - ro.imag, 2 * math.pi)) < 1e-9


def test_two_devices_in_one_process():
    """Handles on devices 0 and 1 in one process: each device gets its own raise of
    the kernels' dynamic shared-memory limits (the fused solve and the DMMA update
    need more than the 48 KB default), so both solve correctly."""
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible devices")
    ddla = _ddla()
    rng = np.random.default_rng(77)
    n, nrhs = 700, 5
    G = rng.standard_normal((n, n))
    A = G @ G.T / n + np.eye(n)
    B = rng.standard_normal((n, nrhs))
    for dev in (0, 1, 0):
        with torch.cuda.device(dev):
            with ddla.Handle(ddla.Backend.GPU) as h:
                dA = ddla.DistributedMatrix.from_global_matrix(h, A, mb=128, nb=128)
                dB = ddla.DistributedMatrix.from_global_matrix(h, B, mb=128, nb=128)
                X, info = ddla.pposv(dA, dB, "L")
                assert info == 0
                Xh = X.to_global_matrix()
        assert np.max(np.abs(A @ Xh - B)) <= 1e-9 * np.max(np.abs(B))
