"""The oracle's phegst (type-1 Hermitian-definite reduction, the consumer of the
Cholesky factor), pinned on the reference test's analytic pair
(tests/generalized_eigen_test_common.h:12-44, tests/test_phegst.cpp:53-155):
B = L L^H with L lower bidiagonal, A = L S L^H with S known, so the reduced
matrix is S; the second pass reduces 1.25 A + 0.37 B to 1.25 S + 0.37 I.  As in
that test, the unused triangles of A and of the factor and the imaginary parts
of A's diagonal hold NaN, the error is relative and scaled by eps * n (<= 400),
the diagonal comes out real and everything past n is left alone."""
import math

import numpy as np
import pytest

from oracle import restated

DT = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}


def _phase(p, i):
    return complex(math.cos(0.23 * i), math.sin(0.23 * i)) if p in "cz" else 1.0


def _eig(i):
    return i - 3.0


def _standard(p, n):
    k = np.arange(n) + 1.0
    norm = float((k * k).sum())
    weighted = float((k * k * np.array([_eig(i) for i in range(n)])).sum())
    S = np.zeros((n, n), dtype=np.complex128)
    for i in range(n):
        for j in range(n):
            x = (_eig(i) if i == j else 0.0) + (i + 1.0) * (j + 1.0) / norm * (
                4 * weighted / norm - 2 * _eig(i) - 2 * _eig(j))
            S[i, j] = x * _phase(p, i) * np.conj(_phase(p, j))
    return S if p in "cz" else S.real


def _bidiagonal(p, n):
    L = np.zeros((n, n), dtype=np.complex128)
    for i in range(n):
        L[i, i] = 1.0 + (i + 1.0) / (n + 1)
        if i:
            L[i, i - 1] = complex(0.17, 0.09) * _phase(p, i) if p in "cz" else 0.17
    return L if p in "cz" else L.real


def _pair(p, n):
    L, S = _bidiagonal(p, n), _standard(p, n)
    return L @ S @ np.conj(L).T, L @ np.conj(L).T, S


@pytest.mark.parametrize("p", list("sdcz"))
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("n", [0, 1, 17, 64])
def test_oracle_phegst_reduces_the_analytic_pair(p, uplo, n):
    A, B, S = _pair(p, n)
    eps = np.finfo(DT[p]).eps
    pad_a, pad_f = 3, 2
    # the factor: the oracle's Cholesky of B, the other triangle poisoned, padding as sentinel
    Fb = np.full((n + pad_f, n + pad_f), 8157.0, dtype=DT[p], order="F")
    Fb[:n, :n] = B.astype(DT[p])
    F, info = restated.potrf(Fb, uplo, n)
    assert info == 0
    F = np.array(F, order="F")
    other = np.triu_indices(n, 1) if uplo == "L" else np.tril_indices(n, -1)
    F[other] = np.nan
    F_before = F.copy()
    for rep in range(2):
        want = S if rep == 0 else 1.25 * S + 0.37 * np.eye(n)
        src = A if rep == 0 else 1.25 * A + 0.37 * B
        Ab = np.full((n + pad_a, n + pad_a), 8157.0, dtype=DT[p], order="F")
        Ab[:n, :n] = src.astype(DT[p])
        Ab[other] = np.nan
        if p in "cz" and n:
            d = np.diag_indices(n)
            Ab.imag[d] = np.nan  # the reference test's NaN imaginary diagonal (real part kept)
        got = restated.phegst(Ab, F, uplo, n)
        if n:
            err = np.abs(got[:n, :n] - want) / np.maximum(np.abs(want), 1.0)
            assert float(err.max()) / (eps * n) <= 400, (p, uplo, n, rep, float(err.max()) / (eps * n))
            assert np.all(np.imag(np.diag(got[:n, :n])) == 0) if p in "cz" else True
            assert np.allclose(got[:n, :n], np.conj(got[:n, :n]).T, rtol=0, atol=0)  # exactly Hermitian
        # rows and columns past n unchanged, the factor untouched
        assert got[n:].tobytes() == Ab[n:].tobytes() and got[:, n:].tobytes() == Ab[:, n:].tobytes()
        assert F.tobytes() == F_before.tobytes()
