"""Bottom-right Cholesky (ddla::potrf_bottom_right / ppotrf_bottom_right):
A = U U^H in the upper triangle ('U') or A = L^H L in the lower one ('L'),
factored from the last column.

* The oracle's restatement of the reference's blocked loop is pinned on the
  reference test's own known-answer construction (tests/test_potrf_bottom_right.cpp:
  a fixed factor, its product, the other triangle and the padding poisoned;
  factor error <= 128 eps n, poisoned entries bit-exact) -- CPU tests.
* The GPU path (C ABI, libddla_c.so) is checked on the same known answers, against
  the oracle on random matrices, on the index of a failed pivot, through the
  descriptor form, and on argument errors -- gpu tests.
"""
import ctypes

import numpy as np
import pytest

from oracle import restated

DT = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}
EPS = {"s": np.finfo(np.float32).eps, "c": np.finfo(np.float32).eps, "d": np.finfo(np.float64).eps,
       "z": np.finfo(np.float64).eps}
KAT_SIZES = [1, 70, 127, 128, 129, 257]


def _selected(uplo, n):
    i, j = np.indices((n, n))
    return (i <= j) if uplo == "U" else (i >= j)


def kat_factor(uplo, n, p):
    """The reference test's factor: diagonal 1.5 + 0.002 (i mod 23), small off-diagonal entries."""
    i, j = np.indices((n, n)).astype(np.float64)
    re = 0.004 * (np.mod(3 * i + 5 * j, 11) - 5)
    F = re.astype(np.complex128)
    if p in "cz":
        F = F + 1j * 0.003 * (np.mod(7 * i + 2 * j, 9) - 4)
    F[np.diag_indices(n)] = 1.5 + 0.002 * np.mod(np.arange(n), 23)
    F[~_selected(uplo, n)] = 0
    return F if p in "cz" else F.real


def kat_input(uplo, n, p, lda):
    """(padded input, expected factor): the product in the selected triangle, the
    reference's marker values in the other triangle and in rows n..lda-1."""
    F = kat_factor(uplo, n, p)
    A = F @ F.conj().T if uplo == "U" else F.conj().T @ F
    i, j = np.indices((n, n)).astype(np.float64)
    other = (-73.0 - 0.013 * i) + (1j * (19.0 + 0.017 * j) if p in "cz" else 0)
    A = np.where(_selected(uplo, n), A, other)
    pad = -911.0 + (37j if p in "cz" else 0)
    host = np.full((lda, n), pad, dtype=DT[p], order="F")
    host[:n, :] = A.astype(DT[p])
    return host, F


def check_kat(uplo, n, p, lda, out, F):
    sel = _selected(uplo, n)
    err = float(np.max(np.abs(out[:n][sel] - F[sel]))) if n else 0.0
    assert err <= 128 * EPS[p] * max(1, n), (p, uplo, n, err)
    ref, _ = kat_input(uplo, n, p, lda)
    np.testing.assert_array_equal(out[:n][~sel], ref[:n][~sel])  # the other triangle, bit for bit
    np.testing.assert_array_equal(out[n:], ref[n:])  # the padding rows, bit for bit


def random_spd(n, p, seed):
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((n, n))
    if p in "cz":
        G = G + 1j * rng.standard_normal((n, n))
    return (G @ G.conj().T / n + np.eye(n)).astype(DT[p])


# ---------------------------------------------------------------- the oracle, on the CPU
@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("n", KAT_SIZES)
def test_oracle_bottom_right_known_answer(p, uplo, n):
    host, F = kat_input(uplo, n, p, n + 3)
    out, info = restated.potrf_bottom_right(host, uplo, n)
    assert info == 0
    check_kat(uplo, n, p, n + 3, out, F)


@pytest.mark.parametrize("uplo", ["U", "L"])
def test_oracle_bottom_right_failed_pivot(uplo):
    """A negative diagonal entry at row r (0-based) of a diagonally dominant matrix
    fails at pivot r + 1: the reversed factorization reaches it after the rows below."""
    n = 300
    for r in (0, 5, 150, 171, 299):
        A = random_spd(n, "d", r) + n * np.eye(n)
        A[r, r] = -1.0
        _, info = restated.potrf_bottom_right(A, uplo)
        assert info == r + 1, (uplo, r, info)


# ---------------------------------------------------------------- the GPU path
def _lib():
    from libddla_b200 import ddla
    return ddla


def _run_gpu(handle, p, uplo, host, n, lda):
    ddla = _lib()
    dA = handle.malloc(host.nbytes)
    try:
        handle.memcpy(dA, host.ctypes.data, host.nbytes)
        info = ddla.potrf_bottom_right(handle, p, uplo, n, dA, lda)
        out = np.empty_like(host)
        handle.memcpy(out.ctypes.data, dA, host.nbytes)
        handle.synchronize()
    finally:
        handle.free(dA)
    return out, info


@pytest.mark.gpu
@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("n", KAT_SIZES)
def test_bottom_right_known_answer(handle, p, uplo, n):
    host, F = kat_input(uplo, n, p, n + 3)
    out, info = _run_gpu(handle, p, uplo, host, n, n + 3)
    assert info == 0
    check_kat(uplo, n, p, n + 3, out, F)


@pytest.mark.gpu
@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("n,pad", [(300, 0), (1025, 5), (2100, 1)])
def test_bottom_right_matches_oracle(handle, p, uplo, n, pad):
    A = random_spd(n, p, 1000 + n)
    host = np.zeros((n + pad, n), dtype=DT[p], order="F")
    host[:n] = A
    out, info = _run_gpu(handle, p, uplo, host, n, n + pad)
    ref, info_ref = restated.potrf_bottom_right(host, uplo, n)
    assert info == info_ref == 0
    sel = _selected(uplo, n)
    err = np.max(np.abs(out[:n][sel] - ref[:n][sel])) / np.max(np.abs(ref[:n][sel]))
    assert err < (2e-5 if p in "sc" else 3e-12), err
    np.testing.assert_array_equal(out[:n][~sel], host[:n][~sel])
    # the factor reproduces A
    Fm = np.where(sel, out[:n], 0).astype(np.complex128)
    prod = Fm @ Fm.conj().T if uplo == "U" else Fm.conj().T @ Fm
    rel = np.max(np.abs(prod - A)) / np.max(np.abs(A))
    assert rel < (1e-5 if p in "sc" else 1e-13), rel


@pytest.mark.gpu
@pytest.mark.parametrize("p", ["d", "z", "s"])
@pytest.mark.parametrize("uplo", ["U", "L"])
def test_bottom_right_failed_pivot(handle, p, uplo):
    n = 700
    for r in (0, 3, 350, 511, 699):
        A = (random_spd(n, p, r) + n * np.eye(n)).astype(DT[p])
        A[r, r] = -1.0
        host = np.asfortranarray(A)
        _, info = _run_gpu(handle, p, uplo, host, n, n)
        _, info_ref = restated.potrf_bottom_right(host, uplo, n)
        assert info == info_ref == r + 1, (p, uplo, r, info, info_ref)


@pytest.mark.gpu
@pytest.mark.parametrize("p", list("dz"))
@pytest.mark.parametrize("uplo", ["U", "L"])
def test_ppotrf_bottom_right_descriptor(handle, p, uplo):
    """The descriptor form factors the leading n x n of a larger described matrix."""
    ddla = _lib()
    n, nd = 257, 300
    host, F = kat_input(uplo, n, p, n)
    M = ddla.DistributedMatrix(handle, nd, nd, mb=64, nb=64, dtype=DT[p], lld=nd + 2)
    full = np.full((M.lld, nd), 5.0, dtype=DT[p], order="F")
    full[:n, :n] = host
    M.from_host(full, full_lld=True)
    info = ctypes.c_int(-1)
    f = getattr(ddla._c_api.lib, f"ddla_{p}_ppotrf_bottom_right")
    ddla._c_api.check_status(f(handle.ptr, uplo.encode(), n, M.data_ptr, M.desc.ctypes.data, ctypes.byref(info)),
                             "ppotrf_bottom_right")
    assert info.value == 0
    out = M.to_host(full_lld=True)
    check_kat(uplo, n, p, n, out[:n, :n], F)
    np.testing.assert_array_equal(out[:, n:], full[:, n:])
    np.testing.assert_array_equal(out[n:, :n], full[n:, :n])


@pytest.mark.gpu
def test_bottom_right_errors(handle):
    ddla = _lib()
    C = ddla._c_api
    info = ctypes.c_int(-1)
    f = C.lib.ddla_d_potrf_bottom_right
    # n = 0: nothing to do, info 0
    assert f(handle.ptr, b"U", 0, None, 1, ctypes.byref(info)) == C.STATUS_SUCCESS and info.value == 0
    for uplo, n, ptr, lda, msg in [(b"X", 4, 256, 4, "uplo must be"), (b"U", -1, 256, 4, "negative matrix size"),
                                   (b"L", 4, None, 4, "null A"), (b"U", 4, 256, 3, "lda too small")]:
        with pytest.raises(C.DdlaError, match=msg):
            C.check_status(f(handle.ptr, uplo, n, ptr, lda, ctypes.byref(info)), "potrf_bottom_right")
    M = ddla.DistributedMatrix(handle, 8, 8, mb=4, nb=4, dtype=np.float64)
    g = C.lib.ddla_d_ppotrf_bottom_right
    with pytest.raises(C.DdlaError, match="invalid triangle, dimensions, blocks or grid"):
        C.check_status(g(handle.ptr, b"U", 9, M.data_ptr, M.desc.ctypes.data, ctypes.byref(info)), "n > M")
    with pytest.raises(C.DdlaError, match="invalid triangle, dimensions, blocks or grid"):
        C.check_status(g(handle.ptr, b"T", 8, M.data_ptr, M.desc.ctypes.data, ctypes.byref(info)), "uplo T")
