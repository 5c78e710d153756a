"""The oracle pinned against the reference tests' known answers, and against real LAPACK (CPU only)."""
import numpy as np
import pytest

import generators as G
from oracle import lapack_arm, restated

TOL_FACTOR = {"s": 2e-5, "c": 2e-5, "d": 3e-12, "z": 3e-12}  # test_ppotrf_grids.cpp:75


@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("n", [1, 2, 17, 38, 129])
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_kat_factor(golden, p, n, uplo):
    A = golden["kat"][f"{p}_{n}_A"]
    L = golden["kat"][f"{p}_{n}_L"]
    F, info = restated.potrf(A, uplo)
    assert info == 0
    want = L if uplo == "L" else L.conj().T
    got = np.tril(F) if uplo == "L" else np.triu(F)
    assert np.max(np.abs(got - want) / (1 + np.abs(want))) < TOL_FACTOR[p]


def test_kat_generator_reproduces_fixture(golden):
    for p, dt in G.DTYPES.items():
        for n in (17, 38):
            np.testing.assert_array_equal(G.kat_matrix(n, dt), golden["kat"][f"{p}_{n}_A"])


@pytest.mark.parametrize("p", ["s", "d"])
@pytest.mark.parametrize("n", [16, 40])
def test_real_spd_solution(golden, p, n):
    z = golden["real_spd"]
    _, X, info = restated.pposv(z[f"{p}_{n}_A"], z[f"{p}_{n}_B"], "L")
    assert info == 0
    tol = 3e-3 if p == "s" else 1e-9  # test_ppotrf_real.cpp:65
    assert np.max(np.abs(X - z[f"{p}_{n}_X"])) < tol


@pytest.mark.parametrize("n", [1, 24])
def test_hpd_solution(golden, n):
    z = golden["hpd"]
    F, X, info = restated.pposv(z[f"z_{n}_A"], z[f"z_{n}_B"], "L")
    assert info == 0
    if n == 1:
        assert abs(F[0, 0] - 2.0) < 1e-12  # test_api_grid_ppotrf.cpp:14-31
    assert np.max(np.abs(X - z[f"z_{n}_X"])) < 5e-9


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_sides_and_triangles(side, uplo):
    rng = np.random.default_rng(3)
    n, nrhs = 23, 4
    M = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    A = M @ M.conj().T + n * np.eye(n)
    X = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    if side == "L":
        B = A @ X
    else:
        X = X.T.copy()
        B = X @ A
    _, Y, info = restated.pposv(A, B, uplo, side)
    assert info == 0
    np.testing.assert_allclose(Y, X, atol=1e-10)


def test_python_cases(golden):
    z = golden["python"]
    A, X = z["ppotrf_ppotrs_A"], z["ppotrf_ppotrs_X"]
    _, Y, info = restated.pposv(A, A @ X, "L")
    assert info == 0 and np.max(np.abs(Y - X)) < 1e-11
    for key in [k for k in z.files if k.startswith("typed_") and k.endswith("_A")]:
        _, k, ch, uplo, _ = key.split("_")
        A, X, B = z[key], z[key[:-1] + "X"], z[key[:-1] + "B"]
        _, Y, info = restated.pposv(A, B, uplo)
        tol = 2e-4 if ch in "fF" else 1e-11  # test_cholesky.py:74
        assert info == 0
        np.testing.assert_allclose(Y, X, atol=tol, rtol=tol)


@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_negative_last_pivot(p, uplo):
    n = 9  # test_cholesky.py:79-92
    A = np.eye(n, dtype=G.DTYPES[p])
    A[-1, -1] = -1
    B = np.ones((n, 2), dtype=A.dtype)
    _, X, info = restated.pposv(A, B, uplo)
    assert info == n
    np.testing.assert_array_equal(X, B)


@pytest.mark.parametrize("p", list("sdcz"))
def test_logdet_cases(golden, p):
    z = golden["logdet"]
    tol = 2e-5 if p in "sc" else 3e-12  # test_diag_logdet.cpp:31-37
    k = 0
    while f"{p}_{k}_diag" in z.files:
        d = z[f"{p}_{k}_diag"]
        A = np.diag(d) if d.size else np.zeros((0, 0), dtype=d.dtype)
        if not bool(z[f"{p}_{k}_valid"]):
            with pytest.raises(ValueError):
                restated.diag_logdet(A)
        else:
            e = z[f"{p}_{k}_expect"]
            r = restated.diag_logdet(A)
            if np.isinf(e[0]):
                assert np.isinf(r.real) and r.real < 0 and r.imag == 0
            else:
                assert abs(r.real - e[0]) < tol * (1 + abs(e[0]))
                assert abs(np.remainder(r.imag - e[1] + np.pi, 2 * np.pi) - np.pi) < tol
        k += 1
    assert k >= 9


def test_logdet_negative_parity_large():
    n = 1025  # test_diag_logdet.cpp:97-103
    A = -np.eye(n)
    r = restated.diag_logdet(A)
    assert abs(r.real) < 1e-12 and abs(r.imag - np.pi) < 1e-12


@pytest.mark.parametrize("p", ["d", "z", "s"])
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_restatement_matches_lapack(p, uplo):
    """The plain-C restatement against the real LAPACK the reference's CPU handle calls."""
    rng = np.random.default_rng(11)
    n, nrhs = 300, 5
    dt = G.DTYPES[p]
    M = rng.standard_normal((n, n))
    if p in "cz":
        M = M + 1j * rng.standard_normal((n, n))
    A = (M @ M.conj().T / n + np.eye(n)).astype(dt)
    B = rng.standard_normal((n, nrhs)).astype(dt)
    F1, X1, i1 = restated.pposv(A, B, uplo)
    F2, X2, i2 = lapack_arm.pposv(A, B, uplo)
    assert i1 == 0 and i2 == 0
    tri = np.tril if uplo == "L" else np.triu
    tol = 1e-4 if p in "sc" else 1e-12
    assert np.max(np.abs(tri(F1) - tri(F2))) < tol * np.max(np.abs(F2))
    assert np.max(np.abs(X1 - X2)) < tol * 10 * np.max(np.abs(X2))
